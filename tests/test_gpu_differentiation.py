"""The differentiation configuration at full size: the two-material porous 64^3 cube
(packing 0.3, m1 = 1.5+0.01i / m2 = 1.7+0.1i at 0.7 / 0.3, seed 11), x = 5, CMRR, CG.

* The GPU adjoint gradient (FP32 FFT matvec, FP64 refinement) of Cabs and M11(180 deg)
  for every dipole against the FP64 reference gradient: the same adjoint formulas with
  every solve in FP64 (ddagpu_solve_fp64, validated against the reference's FP64 build in
  test_gpu_fp64.py).
* The FP64 gradient against central finite differences (step 1e-3 on Re m and Im m) at 32
  seeded dipoles.  A dipole's share of Cabs is about 1e-5 of it, so a difference of 1e-3
  in m moves the observables by about 1e-8 relative, below what a full solve resolves.
  Each perturbed system (m_k -> m_k +- h, a material of its own as a per-dipole reference
  would do, main.cpp:645-677) is therefore solved exactly as p + d: with A p = b the
  converged FP64 solution, A' (p + d) = b' gives A' d = (a'_k - a_k) p_k / a_k at cell k
  alone (b - A p, the same for both signs, cancels in the central difference), and d is
  an FP64 solve to 1e-8 of its right-hand side's discrepancy (the mean residual norm: the
  residual spreads from one cell over all 78,528, so this is about 4e-11 in the 2-norm),
  restarted every 200 steps (COCG stagnates on some of these single-cell systems after a
  near-breakdown step; a restart resets that).
* The cost: the adjoint pass (any combination of the observables) takes at most 2.5x the
  forward pass, in matvecs and in time."""
import time

import numpy as np
import pytest
import torch

from dda_fft_b200.adjoint import GPUBackend, GPUFP64Backend, Problem, observables, porous_target

pytestmark = pytest.mark.gpu


def _grads(P, B, m):
    """[Cabs, M11] and, per observable, the gradient (d/dRe m, d/dIm m) of every dipole."""
    m_re = torch.tensor(m.real, requires_grad=True)
    m_im = torch.tensor(m.imag, requires_grad=True)
    out = []
    for k in range(2):
        m_re.grad = None
        m_im.grad = None
        f = observables(m_re, m_im, P, B)
        f[k].backward()
        out.append(np.stack([m_re.grad.numpy(), m_im.grad.numpy()]))
    return f.detach().numpy(), out


@pytest.fixture(scope="module")
def setup():
    filled, m = porous_target(64, seed=11)
    P = Problem(filled, kd=2 * 5.0 / 64, model="cmrr")
    F = GPUFP64Backend(P, err_max=1e-13)
    f64, g64 = _grads(P, F, m)
    yield P, m, F, f64, g64
    F.close()


def test_gpu_adjoint_matches_fp64_gradient_64(setup):
    P, m, F, f64, g64 = setup
    G = GPUBackend(P, err_max=1e-9)
    fg, gg = _grads(P, G, m)
    G.close()
    assert abs(fg[0] - f64[0]) < 1e-5 * abs(f64[0])
    assert abs(fg[1] - f64[1]) < 1e-4 * abs(f64[1])
    for k in range(2):
        err = np.abs(gg[k] - g64[k]).max() / np.abs(g64[k]).max()
        print(f"observable {k}: GPU adjoint vs FP64 gradient, max error {err:.2e} of the largest "
              f"({P.ndip} dipoles)")
        assert err < 1e-3, (k, err)


def test_fp64_gradient_matches_central_differences_64(setup):
    P, m, F, f64, g64 = setup
    occ, table, a, _ = P.tables(m)
    base = [F.solve(occ, table, P.pinc(a, q)) for q in range(2)]
    rng = np.random.default_rng(32)
    h = 1e-3
    worst = 0.0
    for k in rng.choice(P.ndip, 32, replace=False):
        fd = np.zeros((2, 2))   # [re / im][cabs / m11]
        for part, step in ((0, h), (1, 1j * h)):
            vals = []
            for sgn in (+1, -1):
                mm = m.copy()
                mm[k] += sgn * step
                occ_k, table_k, a_k, _ = P.tables(mm)
                p = []
                for q in range(2):
                    rhs = np.zeros((P.ndip, 3), complex)
                    rhs[k] = (a_k[k] - a[k]) * base[q][k] / a[k]
                    err0 = np.linalg.norm(rhs[k]) / P.ndip          # its discrepancy
                    d = F.solve(occ_k, table_k, rhs, err_max=1e-8 * err0, restart_every=200,
                                restarts=10)
                    assert F.last_err <= 1e-8 * err0
                    p.append(base[q] + d)
                cabs, m11, _ = P.observables(p, a_k)
                vals.append((cabs, m11))
            fd[part] = (np.array(vals[0]) - np.array(vals[1])) / (2 * h)
        for obs in range(2):
            for part in range(2):
                adj = g64[obs][part][k]
                scale = max(abs(fd[part, obs]), np.abs(g64[obs][part]).max() * 1e-3)
                err = abs(adj - fd[part, obs]) / scale
                worst = max(worst, err)
                # the central difference's own O(h^2) error at h = 1e-3 reaches ~1e-4
                assert err < 1e-3, (k, obs, part, adj, fd[part, obs])
    print(f"32 dipoles: FP64 adjoint vs central differences, worst {worst:.2e} of the scale")


def test_adjoint_cost_64():
    filled, m = porous_target(64, seed=11)
    P = Problem(filled, kd=2 * 5.0 / 64, model="cmrr")
    G = GPUBackend(P, err_max=1e-8)
    m_re = torch.tensor(m.real, requires_grad=True)
    m_im = torch.tensor(m.imag, requires_grad=True)
    observables(m_re, m_im, P, G)                        # warm-up
    mv0 = G.matvecs
    t0 = time.perf_counter()
    f = observables(m_re, m_im, P, G)
    t1 = time.perf_counter()
    mv1 = G.matvecs
    (f[0] + 10.0 * f[1]).backward()
    t2 = time.perf_counter()
    mv2 = G.matvecs
    G.close()
    print(f"forward {t1 - t0:.3f} s / {mv1 - mv0} matvecs, backward {t2 - t1:.3f} s / {mv2 - mv1} "
          f"matvecs: {(t2 - t1) / (t1 - t0):.2f}x")
    assert (mv2 - mv1) <= 2.5 * (mv1 - mv0), (mv1 - mv0, mv2 - mv1)
    assert (t2 - t1) <= 2.5 * (t1 - t0), (t1 - t0, t2 - t1)
