"""Adjoint gradients of DDA observables with respect to every dipole's refractive index.

A Python harness over the C ABI (the product host is C++ and has no adjoint): a
torch.autograd.Function whose forward solves both incident polarisations and whose
backward runs one adjoint solve per polarisation through the same matvec.

System (dda_func.cpp:1075-1570): A p = b with A = I - D_a G, b = D_a E_inc, D_a the
per-dipole polarisabilities and G the lattice Green tensor (complex symmetric: every
3x3 block is symmetric and G(r) = G(-r), so G^T = G).  Hence A^T = I - G D_a, and
A^T l = g is solved as A u = D_a g, l = u / a.  With dp/da_k = A^-1 (e_k p_k / a_k)
(b depends on a_k too; p_k / a_k is the local field), an observable f(p, conj p, a)
has the holomorphic derivative

    df/da_k = (partial f / partial a_k) + l_k . p_k / a_k = ... + u_k . p_k / a_k^2,

with g = df/dp (Wirtinger, conj p held fixed), and df/dm_k = df/da_k * a'(m_k).  For a
real f: df/dRe m_k = 2 Re(df/dm_k), df/dIm m_k = -2 Im(df/dm_k).  The gradient is that of
the solved linear system; no solver iterate is stored or differentiated, only the two
converged solutions (the checkpoint of the forward pass).

Observables, as the reference defines them:
  Cabs = 1/2 sum_q 4 pi / |E|^2 sum_k |p_k|^2 (Im a_k / |a_k|^2 - 2/3)  (CabsCext,
         dda_func.cpp:1679-1727, averaged over polarisations as main.cpp:939)
  M11  = 1/2 (|J00|^2 + |J01|^2 + |J10|^2 + |J11|^2) at one scattering direction, the
         Jones matrix of BuildMatrixJones (mmuller.cpp:175-252) from the far fields
         S = sum_k exp(i k.(r_k - c)) p_k, E_sc = S - k (k.S) (dda_func.cpp:1576-1625).
"""
from __future__ import annotations

import numpy as np
import torch

PI = np.pi


def alpha_cm(kd, m):
    """Polarizability_CM, dda_func.cpp:1631-1637."""
    return kd ** 3 * (0.75 / PI) * (m * m - 1) / (m * m + 2)


def dalpha_cm(kd, m):
    return kd ** 3 * (0.75 / PI) * 6 * m / (m * m + 2) ** 2


def alpha_of(model, kd, m):
    """CM or CMRR (dda_func.cpp:1639-1645) and its derivative d alpha / d m."""
    a = alpha_cm(kd, m)
    da = dalpha_cm(kd, m)
    if model == "cm":
        return a, da
    if model == "cmrr":
        den = 1 - (2.0 / 3.0) * 1j * a
        return a / den, da / den ** 2
    raise ValueError(model)


def jones(kinc, ksc, nrm, e0, e1, s0, s1):
    """BuildMatrixJones (mmuller.cpp:175-252) and the derivative of each Jones element
    with respect to the two scattered fields: returns J[2][2], dJ/ds0[2][2][3],
    dJ/ds1[2][2][3]."""
    v = np.cross(kinc, nrm)
    pin = v / np.linalg.norm(v)
    v = np.cross(ksc, nrm)
    psc = -v / np.linalg.norm(v)
    i0n, i1n, i0p, i1p = nrm @ e0, nrm @ e1, pin @ e0, pin @ e1
    den = 1j * (i0n * i1p - i1n * i0p)
    s0n, s1n, s0p, s1p = nrm @ s0, nrm @ s1, psc @ s0, psc @ s1
    J = np.array([[s1p * i0n - s0p * i1n, s0p * i1p - s1p * i0p],
                  [s1n * i0n - s0n * i1n, s0n * i1p - s1n * i0p]]) / den
    d0 = np.array([[-i1n * psc, i1p * psc], [-i1n * nrm, i1p * nrm]]) / den
    d1 = np.array([[i0n * psc, -i0p * psc], [i0n * nrm, -i0p * nrm]]) / den
    return J, d0, d1


class Problem:
    """A lattice target with per-dipole refractive indices, fixed orientation
    (k_inc = z, E = x and y, main.cpp:153-154) and one scattering direction in plane 0."""

    def __init__(self, filled, kd, model="cmrr", theta_deg=180.0):
        self.filled = np.asarray(filled, bool)
        self.grid = self.filled.shape
        self.kd = float(kd)
        self.model = model
        ni, nj, nl = self.grid
        self.idx = np.argwhere(self.filled)                       # active cells
        c = np.array([(ni - 1), (nj - 1), (nl - 1)]) * kd / 2
        self.r = self.idx * kd - c                                 # positions - centre
        self.kinc = np.array([0.0, 0.0, 1.0])
        self.einc = [np.array([1.0, 0, 0], complex), np.array([0, 1.0, 0], complex)]
        th = np.deg2rad(theta_deg)
        self.ksc = np.array([np.sin(th), 0.0, np.cos(th)])
        self.nrm = np.array([0.0, 1.0, 0.0])
        self.ph_inc = np.exp(1j * self.r @ self.kinc)              # exp(i k_inc.(r - c))
        self.ph_sc = np.exp(1j * self.r @ self.ksc)

    @property
    def ndip(self):
        return len(self.idx)

    def tables(self, m):
        """Material table for per-dipole indices m: occupancy with one material per
        distinct value, alpha per material, alpha per dipole and d alpha / d m."""
        vals, inv = np.unique(np.asarray(m, complex), return_inverse=True)
        if len(vals) > 254:
            raise ValueError("at most 254 distinct refractive indices")
        occ = np.zeros(self.grid, np.int8)
        occ[tuple(self.idx.T)] = (inv + 1).astype(np.int8)
        a_mat, da_mat = alpha_of(self.model, self.kd, vals)
        table = np.concatenate([[0.0], a_mat])
        return occ, table, a_mat[inv], da_mat[inv]

    def field(self, per_dipole):
        """(ndip, 3) -> lattice field (ni, nj, nl, 3)."""
        f = np.zeros(self.grid + (3,), complex)
        f[tuple(self.idx.T)] = per_dipole
        return f

    def pinc(self, a, q):
        return (a * self.ph_inc)[:, None] * self.einc[q][None, :]

    def observables(self, p, a):
        """Cabs and M11 from per-dipole moments p[q] (ndip, 3) and alpha a (ndip)."""
        w = a.imag / np.abs(a) ** 2 - 2.0 / 3.0
        cabs = 0.5 * sum(4 * PI * np.sum(np.sum(np.abs(p[q]) ** 2, 1) * w) for q in range(2))
        esc = []
        for q in range(2):
            S = (self.ph_sc[:, None] * p[q]).sum(0)
            esc.append(S - self.ksc * (self.ksc @ S))
        J, _, _ = jones(self.kinc, self.ksc, self.nrm, self.einc[0], self.einc[1], esc[0], esc[1])
        m11 = 0.5 * np.sum(np.abs(J) ** 2)
        return cabs, m11, esc

    def sources(self, p, a, w_cabs, w_m11):
        """Adjoint sources g[q] = w_cabs dCabs/dp[q] + w_m11 dM11/dp[q] (Wirtinger) and the
        explicit derivative of w_cabs Cabs with respect to alpha."""
        w = a.imag / np.abs(a) ** 2 - 2.0 / 3.0
        _, _, esc = self.observables(p, a)
        J, d0, d1 = jones(self.kinc, self.ksc, self.nrm, self.einc[0], self.einc[1], esc[0], esc[1])
        g = []
        for q, dq in ((0, d0), (1, d1)):
            v = 0.5 * np.einsum("ab,abc->c", np.conj(J), dq)      # dM11/dEsc_q
            v = v - self.ksc * (self.ksc @ v)                     # projector is symmetric
            gq = w_cabs * 0.5 * 4 * PI * np.conj(p[q]) * w[:, None]
            gq = gq + w_m11 * self.ph_sc[:, None] * v[None, :]
            g.append(gq)
        # d/da of Im(a)/|a|^2 = -Im(1/a): -i / (2 a^2)
        direct = w_cabs * 0.5 * sum(4 * PI * np.sum(np.abs(p[q]) ** 2, 1) for q in range(2)) * (
            -0.5j / a ** 2)
        return g, direct


class GPUBackend:
    """Solves through libddagpu (FP32 matvec, FP64 refinement)."""

    def __init__(self, problem: Problem, err_max=1e-9, solver=0):
        import dda_fft_b200 as D
        self.P = problem
        self.ctx = D.Context(problem.grid, problem.kd, max_rhs=1)
        self.err_max = err_max
        self.solver = solver
        self.matvecs = 0

    def solve(self, occ, table, rhs_dipoles):
        mv = np.array([0] + [1] * (len(table) - 1), np.int32)
        x, info = self.ctx.solve_linear(occ, table, mv, self.P.field(rhs_dipoles), solver=self.solver,
                                        err_max=self.err_max, max_step=60, refine=True)
        self.matvecs += info["matvecs"]
        return x[tuple(self.P.idx.T)].astype(complex)

    def close(self):
        self.ctx.close()


class GPUFP64Backend:
    """FP64 solves on the GPU (ddagpu_solve_fp64: fields, FFTs and scalars in double, the
    reference's CG recurrences), for reference gradients and finite differences at sizes
    the CPU oracle cannot reach.  x0 (per-dipole start) continues from a nearby solution."""

    def __init__(self, problem: Problem, err_max=1e-13, solver=0, max_step=5000):
        import dda_fft_b200 as D
        self.P = problem
        self.ctx = D.Context(problem.grid, problem.kd, max_rhs=1)
        self.err_max = err_max
        self.solver = solver
        self.max_step = max_step
        self.matvecs = 0
        self.last_err = 0.0

    def solve(self, occ, table, rhs_dipoles, x0=None, err_max=None, restart_every=None,
              restarts=0):
        """With restart_every, CG runs at most that many steps at a time and restarts from
        its best iterate (a fresh search direction), up to `restarts` times: COCG can
        stagnate after a near-breakdown step, and a restart resets that."""
        mv = np.array([0] + [1] * (len(table) - 1), np.int32)
        target = self.err_max if err_max is None else err_max
        steps = self.max_step if restart_every is None else restart_every
        x = None if x0 is None else self.P.field(x0)
        for _ in range(restarts + 1):
            r = self.ctx.solve_fp64(occ, table, mv, self.P.kd, self.P.kinc, self.P.einc[0], None,
                                    solver=self.solver, max_step=steps, err_max=target,
                                    rhs=self.P.field(rhs_dipoles), x0=x, want_p=True, trace=False)
            self.matvecs += r["matvecs"]
            self.last_err = min(r["err"], r["err_min"])
            x = r["p"]
            if self.last_err <= target:
                break
        return x[tuple(self.P.idx.T)]

    def close(self):
        self.ctx.close()


class OracleBackend:
    """FP64 solves of the oracle (test infrastructure; for reference gradients)."""

    def __init__(self, problem: Problem, oracle, err_max=1e-13, solver=0):
        self.P = problem
        self.O = oracle
        self.ahat = oracle.green_hat(*problem.grid, problem.kd)
        self.err_max = err_max
        self.solver = solver

    def solve(self, occ, table, rhs_dipoles):
        mv = np.array([0] + [1] * (len(table) - 1), np.int32)
        r = self.O.dda_fft(occ, table, mv, self.P.kd, self.P.kinc, self.P.einc[0], self.ahat,
                           np.zeros((1, 1, 3)), solver=self.solver, max_step=4000,
                           err_max=self.err_max, rhs=self.P.field(rhs_dipoles))
        return r["p"][tuple(self.P.idx.T)]

    def close(self):
        pass


class DDAObservables(torch.autograd.Function):
    """(Re m, Im m) per dipole -> [Cabs, M11]; backward by one adjoint solve per
    polarisation."""

    @staticmethod
    def forward(ctx, m_re, m_im, problem, backend):
        m = m_re.detach().cpu().numpy() + 1j * m_im.detach().cpu().numpy()
        occ, table, a, da = problem.tables(m)
        p = [backend.solve(occ, table, problem.pinc(a, q)) for q in range(2)]
        cabs, m11, _ = problem.observables(p, a)
        ctx.problem, ctx.backend = problem, backend
        ctx.state = (occ, table, a, da, p)
        return torch.tensor([cabs, m11], dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_out):
        P, B = ctx.problem, ctx.backend
        occ, table, a, da, p = ctx.state
        w_cabs, w_m11 = (float(v) for v in grad_out)
        g, direct = P.sources(p, a, w_cabs, w_m11)
        dfda = direct.copy()
        for q in range(2):
            u = B.solve(occ, table, a[:, None] * g[q])            # A u = D_a g
            dfda = dfda + np.sum(u * p[q], 1) / a ** 2
        dfdm = dfda * da
        return (torch.from_numpy(2 * dfdm.real), torch.from_numpy(-2 * dfdm.imag), None, None)


def observables(m_re, m_im, problem, backend):
    return DDAObservables.apply(m_re, m_im, problem, backend)


def porous_target(n, packing=0.3, frac1=0.7, seed=11, m1=1.5 + 0.01j, m2=1.7 + 0.1j):
    """Two-material porous cube: each cell filled with probability `packing`, material 1
    or 2 with probability frac1 / 1 - frac1 (seeded)."""
    rng = np.random.default_rng(seed)
    filled = rng.random((n, n, n)) < packing
    mat = rng.random((n, n, n)) < frac1
    m = np.where(mat, m1, m2)[filled]
    return filled, m
