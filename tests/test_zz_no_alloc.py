"""The allocation-free far field (ddagpu_farfield_noalloc) against the context-based one.

Some callers cannot allocate device memory -- code recorded into a CUDA graph, loops
that forbid allocator calls, hosts that only hand out pre-allocated buffers -- so this
entry point keeps its FP64 accumulators in a fixed device array of the library instead.
The test calls it twice in a row through the C ABI (the second call must not see the
first call's sums) and compares both with ddagpu_farfield, under the same tolerance as
the far-field parity test.  Collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ellipsoid(n):
    c = n / 2 - 0.5
    g = np.arange(n) - c
    r = (g[:, None, None] ** 2 / (n / 2) ** 2 + g[None, :, None] ** 2 / (0.35 * n) ** 2
         + g[None, None, :] ** 2 / (0.25 * n) ** 2)
    return (r <= 1.0).astype(np.int8)


def test_farfield_noalloc_matches_context_farfield():
    import torch
    import dda_fft_b200 as D
    L = D.lib()
    n, kd, ndir = 32, 0.375, 3 * 19
    rng = np.random.default_rng(17)
    occ = _ellipsoid(n)
    mv = np.array([0, 1], np.int32)
    th = np.deg2rad(np.arange(19) * 10.0)
    ksc = np.concatenate([np.stack([np.cos(a) * np.sin(th), -np.sin(a) * np.sin(th), np.cos(th)], 1)
                          for a in np.deg2rad([0.0, 60.0, 120.0])]).astype(np.float32)
    with D.Context(n, kd) as ctx:
        outs = []
        for call in range(2):
            p = (rng.standard_normal((n, n, n, 3)) + 1j * rng.standard_normal((n, n, n, 3))).astype(np.complex64)
            ref = ctx.farfield(occ, mv, kd, p, ksc)
            dev = torch.device("cuda", 0)
            occ_d = torch.from_numpy(occ).to(dev)
            mv_d = torch.from_numpy(mv).to(dev)
            p_d = torch.from_numpy(np.ascontiguousarray(np.moveaxis(p, 3, 0))).to(dev)
            k_d = torch.from_numpy(ksc).to(dev)
            e_d = torch.zeros(ndir * 6, dtype=torch.float32, device=dev)
            stream = torch.cuda.current_stream(dev)
            rc = L.ddagpu_farfield_noalloc(0, n, n, n, kd, C.c_void_p(occ_d.data_ptr()),
                                           C.c_void_p(mv_d.data_ptr()), len(mv) - 1,
                                           C.c_void_p(p_d.data_ptr()),
                                           ndir, C.c_void_p(k_d.data_ptr()), C.c_void_p(e_d.data_ptr()),
                                           C.c_void_p(stream.cuda_stream))
            assert rc == 0, L.ddagpu_last_error()
            stream.synchronize()
            got = e_d.cpu().numpy().view(np.complex64).reshape(ndir, 3)
            err = np.abs(got - ref).max() / np.abs(ref).max()
            assert err < 1e-5, (call, err)
            outs.append(got)
        assert np.abs(outs[0] - outs[1]).max() > 0     # different inputs, independent results


def test_farfield_noalloc_rejects_too_many_directions():
    import dda_fft_b200 as D
    L = D.lib()
    rc = L.ddagpu_farfield_noalloc(0, 16, 16, 16, 0.5, C.c_void_p(1), C.c_void_p(1), 1, C.c_void_p(1),
                                   8193, C.c_void_p(1), C.c_void_p(1), None)
    assert rc == -1
    assert b"8192" in L.ddagpu_last_error()


def test_small_noalloc_call_keeps_a_large_context_working():
    """A call on a small lattice between two far fields of a 128^3 context: the kernels'
    shared-memory limits are per process, so the small call must not lower what the large
    context needs."""
    import torch
    import dda_fft_b200 as D
    L = D.lib()
    rng = np.random.default_rng(5)
    big, small, kd = 128, 16, 0.25
    occ_b = _ellipsoid(big)
    mv = np.array([0, 1], np.int32)
    ksc = np.array([[0.0, 0.0, 1.0], [0.6, 0.0, 0.8], [0.0, 0.0, -1.0]], np.float32)
    p_b = (rng.standard_normal((big, big, big, 3)) + 1j * rng.standard_normal((big, big, big, 3))).astype(np.complex64)
    with D.Context(big, kd) as ctx:
        first = ctx.farfield(occ_b, mv, kd, p_b, ksc)
        dev = torch.device("cuda", 0)
        occ_s = torch.from_numpy(_ellipsoid(small)).to(dev)
        mv_d = torch.from_numpy(mv).to(dev)
        p_s = torch.zeros((3, small, small, small), dtype=torch.complex64, device=dev)
        k_d = torch.from_numpy(ksc).to(dev)
        e_d = torch.zeros(3 * 6, dtype=torch.float32, device=dev)
        rc = L.ddagpu_farfield_noalloc(0, small, small, small, kd, C.c_void_p(occ_s.data_ptr()),
                                       C.c_void_p(mv_d.data_ptr()), 1, C.c_void_p(p_s.data_ptr()), 3,
                                       C.c_void_p(k_d.data_ptr()), C.c_void_p(e_d.data_ptr()), None)
        assert rc == 0, L.ddagpu_last_error()
        torch.cuda.synchronize()
        with D.Context(small, kd) as _:   # a small context created after the large one
            pass
        again = ctx.farfield(occ_b, mv, kd, p_b, ksc)
        assert np.array_equal(first, again)


def test_noalloc_ignores_material_indices_beyond_n_mat():
    """Cells whose material index exceeds n_mat count as empty: the activity flags are never
    read past n_mat."""
    import torch
    import dda_fft_b200 as D
    L = D.lib()
    n, kd = 16, 0.5
    rng = np.random.default_rng(9)
    occ = _ellipsoid(n)
    occ2 = occ.copy()
    occ2[occ2 == 1] = rng.choice(np.array([1, 7], np.int8), size=int((occ2 == 1).sum()))
    dev = torch.device("cuda", 0)
    p = (rng.standard_normal((3, n, n, n)) + 1j * rng.standard_normal((3, n, n, n))).astype(np.complex64)
    p_d = torch.from_numpy(p).to(dev)
    mv_d = torch.tensor([0, 1], dtype=torch.int32, device=dev)
    ksc = np.array([[0.0, 0.0, 1.0], [0.0, 0.6, 0.8]], np.float32)
    k_d = torch.from_numpy(ksc).to(dev)
    outs = []
    for o in (np.where(occ2 == 7, 0, occ2).astype(np.int8), occ2):
        o_d = torch.from_numpy(np.ascontiguousarray(o)).to(dev)
        e_d = torch.zeros(2 * 6, dtype=torch.float32, device=dev)
        rc = L.ddagpu_farfield_noalloc(0, n, n, n, kd, C.c_void_p(o_d.data_ptr()), C.c_void_p(mv_d.data_ptr()),
                                       1, C.c_void_p(p_d.data_ptr()), 2, C.c_void_p(k_d.data_ptr()),
                                       C.c_void_p(e_d.data_ptr()), None)
        assert rc == 0, L.ddagpu_last_error()
        torch.cuda.synchronize()
        outs.append(e_d.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])
