"""Adjoint gradients on the GPU (libddagpu solves, FP64 refinement) against the FP64
oracle's adjoint gradient for every dipole, and the cost of the backward pass."""
import time

import numpy as np
import pytest
import torch

from dda_fft_b200.adjoint import GPUBackend, OracleBackend, Problem, observables, porous_target

pytestmark = pytest.mark.gpu


def _grads(P, B, m):
    m_re = torch.tensor(m.real, requires_grad=True)
    m_im = torch.tensor(m.imag, requires_grad=True)
    f = observables(m_re, m_im, P, B)
    out = []
    for k in range(2):
        if m_re.grad is not None:
            m_re.grad = None
            m_im.grad = None
        f = observables(m_re, m_im, P, B)
        f[k].backward()
        out.append(np.concatenate([m_re.grad.numpy(), m_im.grad.numpy()]))
    return f.detach().numpy(), out


def test_gpu_adjoint_matches_fp64_gradient(oracle):
    filled, m = porous_target(16, seed=11)
    P = Problem(filled, kd=2 * 5.0 / 64, model="cmrr")       # the 64^3, x = 5 lattice spacing
    G = GPUBackend(P, err_max=1e-9)
    O = OracleBackend(P, oracle, err_max=1e-13)
    fg, gg = _grads(P, G, m)
    fo, go = _grads(P, O, m)
    assert abs(fg[0] - fo[0]) < 1e-5 * abs(fo[0])
    assert abs(fg[1] - fo[1]) < 1e-4 * abs(fo[1])
    for k in range(2):
        err = np.abs(gg[k] - go[k]).max() / np.abs(go[k]).max()
        assert err < 1e-3, (k, err)
    G.close()


def test_gpu_adjoint_cost():
    """Backward (one adjoint solve per polarisation, any combination of the observables)
    against the forward pass (one solve per polarisation): at most 2.5x."""
    filled, m = porous_target(32, seed=11)
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
    assert (mv2 - mv1) <= 2.5 * (mv1 - mv0), (mv1 - mv0, mv2 - mv1)
    assert (t2 - t1) <= 2.5 * (t1 - t0) + 0.05, (t1 - t0, t2 - t1)
    assert np.isfinite(m_re.grad.numpy()).all() and np.abs(m_im.grad.numpy()).max() > 0
    G.close()
