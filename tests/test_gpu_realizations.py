"""Realisation batches: right-hand sides of one batched solve with different occupancies
(random / agglomerate targets, main.cpp:806-985 where the target changes per sample).
Checked against the FP64 oracle's sample loop run on each realisation alone, against the
single-occupancy batch, and -- for agglomerates rasterised on the GPU -- against the
reference generator's occupancies."""
import os

import numpy as np
import pytest

from pyoracle import orientation_solves

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def D():
    import dda_fft_b200
    return dda_fft_b200


@pytest.fixture(scope="module")
def fx():
    return np.load(os.path.join(ROOT, "tests", "golden", "targets_v72.npz"))


def targets(oracle, n):
    """Five different 16^3 occupancies: ellipsoids of several aspect ratios, a random
    porous cube and a two-material cube."""
    out = []
    for ba, ca in ((1.0, 1.0), (0.7, 0.5), (0.5, 0.9)):
        occ, _ = oracle.gen_ellipsoid(n, n, n, ba, ca)
        out.append(occ)
    rng = np.random.default_rng(3)
    out.append((rng.random((n, n, n)) < 0.4).astype(np.int8))
    two = np.ones((n, n, n), np.int8)
    two[: n // 2] = 2
    out.append(two)
    return out


def check(r, k, o, mtol=1e-3):
    for q in ("cabs", "cext"):
        assert abs(r[q][k] - o[q]) <= 1e-4 * abs(o[q]), (q, k, r[q][k], o[q])
    M, Mo = r["mueller"][k].ravel(), o["mueller"].ravel()
    sig = np.abs(Mo) > 1e-3 * np.abs(Mo).max()
    assert (np.abs(M[sig] - Mo[sig]) / np.abs(Mo[sig])).max() < mtol


@pytest.mark.parametrize("max_rhs", [2, 4, 16])
def test_realizations_vs_oracle(D, oracle, max_rhs):
    """Each realisation of a batch (chunked by max_rhs / 2) equals the FP64 sample loop on
    that occupancy alone; two materials, CG, fixed orientation."""
    n, x = 16, 3.0
    mats = [(1.5, 0.01), (1.7, 0.1)]
    occs = targets(oracle, n)
    cfg = D.BatchConfig(occ=None, materials=mats, nplanes=2, err_max=1e-4, max_step=60)
    with D.Context(n, 2 * x / n, max_rhs=max_rhs) as ctx:
        r = ctx.realization_solves(cfg, np.stack(occs))
    assert r["n_rhs"] == 2 * len(occs)
    for k, occ in enumerate(occs):
        o = orientation_solves(oracle, n, x, mats, 1, occ=occ, nplanes=2, err_max=1e-4,
                               max_step=60)
        check(r, k, o)


def test_realizations_equal_single_occupancy_batches(D, oracle):
    """A realisation batch with rotations equals, realisation by realisation, the
    orientation batch of that one occupancy (BiCGStab, LDR: per-polarisation alpha)."""
    n, x = 16, 2.5
    occs = targets(oracle, n)[:4]
    rot = D.mc_rotations(7, len(occs))
    cfg = D.BatchConfig(occ=None, materials=[(1.55, 0.005)], solver=2, polarizability=5,
                        max_step=100, err_max=1e-4)
    with D.Context(n, 2 * x / n, max_rhs=4) as ctx:
        r = ctx.realization_solves(cfg, np.stack(occs), rot)
        for k, occ in enumerate(occs):
            cfg1 = D.BatchConfig(occ=occ, materials=[(1.55, 0.005)], solver=2, polarizability=5,
                                 max_step=100, err_max=1e-4)
            s = ctx.orientation_solves(cfg1, rot[k:k + 1])
            for q in ("cabs", "cext"):
                assert abs(r[q][k] - s[q][0]) <= 1e-5 * abs(s[q][0])
            assert np.abs(r["mueller"][k] - s["mueller"][0]).max() <= 1e-5 * np.abs(s["mueller"][0]).max()


def test_realization_without_dipoles_is_rejected(D):
    n = 8
    occs = np.ones((2, n, n, n), np.int8)
    occs[1] = 0
    cfg = D.BatchConfig(occ=None, materials=[(1.5, 0.01)])
    with D.Context(n, 0.5, max_rhs=4) as ctx:
        with pytest.raises(D.DDAGPUError):
            ctx.realization_solves(cfg, occs)
        bad = np.ones((1, n, n, n), np.int8) * 3
        with pytest.raises(D.DDAGPUError):
            ctx.realization_solves(cfg, bad)


@pytest.mark.parametrize("name", ["c3b32", "caps64"])
def test_agglomerate_solves(D, oracle, fx, name):
    """Agglomerates rasterised on the GPU into the batch equal the realisation batch of the
    reference generator's occupancies; the first one is checked against the FP64 oracle."""
    n, r_m, lr, _, seed, count = fx[f"{name}_cfg"]
    n, count = int(n), int(count)
    x = 2.0
    a = D.Agglomerate(state=int(seed))
    mons = [a.place(n, float(r_m), float(r_m * lr), count) for _ in range(3)]
    np.testing.assert_array_equal(mons[0], fx[f"{name}_monomers"])
    occs = np.stack([D.Agglomerate.rasterize((n, n, n), m)[0] for m in mons])
    ref0 = np.unpackbits(fx[f"{name}_occ_bits"])[: n ** 3].reshape(n, n, n)
    np.testing.assert_array_equal(occs[0], ref0)
    cfg = D.BatchConfig(occ=None, materials=[(1.55, 0.005)], err_max=1e-4, max_step=60)
    with D.Context(n, 2 * x / n, max_rhs=4) as ctx:
        g = ctx.agglomerate_solves(cfg, mons)
        h = ctx.realization_solves(cfg, occs)
    assert list(g["ndip"]) == [int((o != 0).sum()) for o in occs]
    assert g["ndip"][0] == int(fx[f"{name}_ndip_next"][0])
    for q in ("cabs", "cext"):
        np.testing.assert_allclose(g[q], h[q], rtol=1e-5)
    np.testing.assert_allclose(g["mueller"], h["mueller"], rtol=1e-5,
                               atol=1e-6 * np.abs(h["mueller"]).max())
    if n <= 32:
        o = orientation_solves(oracle, n, x, [(1.55, 0.005)], 1, occ=occs[0], err_max=1e-4,
                               max_step=60)
        check(g, 0, o)


def test_agglomerate_sample_loop_vs_reference(D, oracle, fx):
    """The reference's sample loop on agglomerates (32^3, x = 6, m = 1.55+0.005i, CM, CG,
    3 realisations drawn one after another by worker 0 of seed 7): our placement on the
    same stream, GPU rasterisation and one batched solve; sums against the FP64 oracle on
    the same occupancies and the float reference's own sums."""
    n, x, mat = 32, 6.0, (1.55, 0.005)
    count = D.Agglomerate.count((n, n, n), 0.25, 3.0, 0.0)
    a = D.Agglomerate(base_seed=7, worker=0)
    mons = [a.place(n, 3.0, 0.0, count) for _ in range(3)]
    cfg = D.BatchConfig(occ=None, materials=[mat])
    with D.Context(n, 2 * x / n, max_rhs=6) as ctx:
        g = ctx.agglomerate_solves(cfg, mons)
    occs = [D.Agglomerate.rasterize((n, n, n), m)[0] for m in mons]
    o = [orientation_solves(oracle, n, x, [mat], 1, occ=occ) for occ in occs]
    ref = fx["agg32_loop3"]
    for k, q in ((0, "cabs"), (1, "cext")):
        r64 = sum(v[q] for v in o)
        gate = max(1e-4 * abs(r64), 2 * abs(ref[k] - r64))
        assert abs(g[q].sum() - r64) <= gate, (q, g[q].sum(), ref[k], r64)
    M = g["mueller"].sum(axis=0).ravel()
    M64 = sum(v["mueller"] for v in o).ravel()
    sig = np.abs(M64) > 1e-3 * np.abs(M64).max()
    assert (np.abs(M[sig] - M64[sig]) / np.abs(M64[sig])).max() < 1e-3
    sig = np.abs(ref[2:]) > 1e-3 * np.abs(ref[2:]).max()
    assert (np.abs(M[sig] - ref[2:][sig]) / np.abs(ref[2:][sig])).max() < 3e-3


@pytest.mark.parametrize("grid,solver", [((32, 16, 32), 2), ((8, 16, 4), 0), ((16, 32, 16), 1)])
def test_rectangular_batches_vs_oracle(D, oracle, grid, solver):
    """Batched Monte-Carlo orientations on rectangular lattices (specialised passes for
    32 x 16 x 32 and 16 x 32 x 16, generic passes for 8 x 16 x 4) with BiCGStab, CG and AA*
    against the FP64 sample loop, summed over 3 orientations; two planes."""
    occ, _ = oracle.gen_ellipsoid(*grid, 0.5 if grid[1] < grid[0] else 1.0,
                                  1.0 if grid[2] >= grid[0] else 0.5)
    x = 0.125 * grid[0]
    cfg = D.BatchConfig(occ=occ, materials=[(1.5, 0.02)], solver=solver, err_max=1e-4,
                        max_step=200, nplanes=2)
    with D.Context(grid, 2 * x / grid[0], max_rhs=4) as ctx:
        r = ctx.orientation_solves(cfg, D.mc_rotations(11, 3))
    o = orientation_solves(oracle, grid, x, [(1.5, 0.02)], 3,
                           b_a=0.5 if grid[1] < grid[0] else 1.0,
                           c_a=1.0 if grid[2] >= grid[0] else 0.5, target=2, solver=solver,
                           err_max=1e-4, max_step=200, nplanes=2, orientation=1, seed=11, occ=occ)
    for q in ("cabs", "cext"):
        assert abs(r[q].sum() - o[q]) <= 1e-4 * abs(o[q]), (q, r[q].sum(), o[q])
    M, Mo = r["mueller"].sum(axis=0).ravel(), o["mueller"].ravel()
    sig = np.abs(Mo) > 1e-3 * np.abs(Mo).max()
    assert (np.abs(M[sig] - Mo[sig]) / np.abs(Mo[sig])).max() < 1e-3


def test_realizations_far_field_by_kz_groups(D, oracle):
    """Realisations of different occupancies (fixed orientation, 12 scattering planes of 37
    angles: 37 distinct kz, 12 directions each) with the far field by kz groups (mode 2,
    each realisation's pair of right-hand sides reading its own occupancy) and by direction
    (mode 1): equal to FP32 rounding, and each realisation against the FP64 sample loop."""
    n, x = 16, 3.0
    mats = [(1.5, 0.01), (1.7, 0.1)]
    occs = targets(oracle, n)
    cfg = D.BatchConfig(occ=None, materials=mats, nplanes=12, theta_step=5.0, err_max=1e-4,
                        max_step=60)
    res = {}
    with D.Context(n, 2 * x / n, max_rhs=16) as ctx:
        for mode in (1, 2):
            ctx.set_farfield_mode(mode)
            res[mode] = ctx.realization_solves(cfg, np.stack(occs))
    for q in ("cabs", "cext"):
        assert np.array_equal(res[1][q], res[2][q]) or \
            (np.abs(res[1][q] - res[2][q]) / np.abs(res[1][q])).max() < 1e-6, q
    M1, M2 = res[1]["mueller"], res[2]["mueller"]
    sig = np.abs(M1) > 1e-3 * np.abs(M1).max()
    assert (np.abs(M2 - M1)[sig] / np.abs(M1)[sig]).max() < 1e-5
    for k, occ in enumerate(occs):
        o = orientation_solves(oracle, n, x, mats, 1, occ=occ, nplanes=12, theta_step=5.0,
                               err_max=1e-4, max_step=60)
        check(res[2], k, o)
