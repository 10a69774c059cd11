"""The adjoint formulas of dda_fft_b200/adjoint.py checked with FP64 oracle solves (no GPU):
the adjoint gradient of Cabs and M11(180 deg) against central finite differences
(step 1e-3 on Re m and Im m of single dipoles, each perturbed dipole a material of its
own, as a per-dipole reference would do)."""
import numpy as np
import torch

from dda_fft_b200.adjoint import OracleBackend, Problem, observables, porous_target


def fd_gradient(P, B, m, k, h=1e-3):
    out = np.zeros((2, 2))   # [re/im][cabs/m11]
    for part, step in ((0, h), (1, 1j * h)):
        vals = []
        for s in (+1, -1):
            mm = m.copy()
            mm[k] += s * step
            occ, table, a, _ = P.tables(mm)
            p = [B.solve(occ, table, P.pinc(a, q)) for q in range(2)]
            cabs, m11, _ = P.observables(p, a)
            vals.append((cabs, m11))
        out[part] = (np.array(vals[0]) - np.array(vals[1])) / (2 * h)
    return out


def test_fp64_adjoint_matches_finite_differences(oracle):
    filled, m = porous_target(8, seed=11)
    P = Problem(filled, kd=0.35, model="cmrr")
    B = OracleBackend(P, oracle, err_max=1e-13)
    m_re = torch.tensor(m.real, requires_grad=True)
    m_im = torch.tensor(m.imag, requires_grad=True)
    grads = []
    for w in ((1.0, 0.0), (0.0, 1.0)):
        f = observables(m_re, m_im, P, B)
        (f[0] * w[0] + f[1] * w[1]).backward()
        grads.append((m_re.grad.numpy().copy(), m_im.grad.numpy().copy()))
        m_re.grad = None
        m_im.grad = None
    rng = np.random.default_rng(4)
    for k in rng.choice(P.ndip, 6, replace=False):
        fd = fd_gradient(P, B, m, k)
        for obs in range(2):
            for part in range(2):
                adj = grads[obs][part][k]
                scale = max(abs(fd[part, obs]), np.abs(grads[obs][part]).max() * 1e-3)
                assert abs(adj - fd[part, obs]) < 2e-4 * scale, (k, obs, part, adj, fd[part, obs])
