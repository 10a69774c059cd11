"""Agglomerate targets (iGenerateAnthrax, particle.cpp:21-85) against the reference's own
generator: the host placement and its random stream must reproduce the reference's
monomers and next draw bit for bit (CPU tests), and the GPU rasterisation the reference's
occupancy cell for cell (GPU tests).  Fixtures: tests/golden/targets_v72.npz, written by
tests/golden/make_golden.py from the reference's compiled sources."""
import hashlib
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CASES = ["c3b32", "c3b64", "caps64", "c3b128"]


@pytest.fixture(scope="module")
def fx():
    return np.load(os.path.join(ROOT, "tests", "golden", "targets_v72.npz"))


def cfg(fx, name):
    n, r, lr, rho, seed, count = fx[f"{name}_cfg"]
    return int(n), float(r), float(lr), float(rho), int(seed), int(count)


def next_draw(state):
    """one xorshift64* draw (randomize.cpp:51-58), for checking where the stream stopped"""
    m = (1 << 64) - 1
    s = state
    s ^= s >> 12
    s = (s ^ (s << 25)) & m
    s ^= s >> 27
    return ((s * 2685821657736338717) & m) >> 33


@pytest.mark.parametrize("name", CASES)
def test_monomer_count(fx, name):
    from dda_fft_b200 import Agglomerate
    n, r, lr, rho, _, count = cfg(fx, name)
    assert Agglomerate.count((n, n, n), rho, r, lr) == count


@pytest.mark.parametrize("name", CASES)
def test_placement_matches_reference(fx, name):
    from dda_fft_b200 import Agglomerate
    n, r, lr, _, seed, count = cfg(fx, name)
    a = Agglomerate(state=seed)
    mon = a.place(n, r, r * lr, count)
    np.testing.assert_array_equal(mon, fx[f"{name}_monomers"])
    assert next_draw(a.state) == int(fx[f"{name}_ndip_next"][1])


def test_rng_seed_per_worker(oracle):
    """dda_srand(base + golden-ratio step x (worker + 1)), main.cpp:803-804: the stream
    of worker w is the one the oracle's Monte-Carlo draws start from."""
    from dda_fft_b200 import Agglomerate, lib
    for base, w in ((7, 0), (7, 3), (0, 0), (123456789, 15)):
        s = int(lib().ddagpu_rng_seed(base, w))
        assert s == (base + 0x9E3779B97F4A7C15 * (w + 1)) % (1 << 64) or s == 0x9E3779B97F4A7C15
        assert Agglomerate(base, w).state == s
        assert next_draw(s) == int(oracle.rng(s, 1)[0])


def test_placement_rejects_bad_arguments():
    from dda_fft_b200 import Agglomerate, DDAGPUError
    with pytest.raises(DDAGPUError):
        Agglomerate(state=1).place(32, 0.0, 0.0, 4)
    with pytest.raises(DDAGPUError):            # cannot fit: placement gives up, no hang
        Agglomerate(state=1).place(8, 3.5, 0.0, 50)


def test_stream_continues_across_samples(fx):
    """Two samples drawn one after the other from one state equal the reference's first
    sample, then a sample started from where it stopped."""
    from dda_fft_b200 import Agglomerate
    n, r, lr, _, seed, count = cfg(fx, "c3b32")
    a = Agglomerate(state=seed)
    first = a.place(n, r, r * lr, count)
    mid = a.state
    second = a.place(n, r, r * lr, count)
    np.testing.assert_array_equal(first, fx["c3b32_monomers"])
    np.testing.assert_array_equal(second, Agglomerate(state=mid).place(n, r, r * lr, count))
    assert not np.array_equal(first, second)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_rasterization_matches_reference(fx, name):
    from dda_fft_b200 import Agglomerate
    n, r, lr, _, seed, count = cfg(fx, name)
    occ, nd, mon = Agglomerate(state=seed).generate((n, n, n), r, r * lr, count)
    np.testing.assert_array_equal(mon, fx[f"{name}_monomers"])
    assert nd == int(fx[f"{name}_ndip_next"][0])
    assert int((occ != 0).sum()) == nd
    assert set(np.unique(occ)) <= {0, 1}
    filled = (occ != 0).astype(np.uint8)
    if f"{name}_occ_bits" in fx:
        ref = np.unpackbits(fx[f"{name}_occ_bits"])[: n ** 3].reshape(n, n, n)
        np.testing.assert_array_equal(filled, ref)
    digest = np.frombuffer(hashlib.sha256(filled.tobytes()).digest(), np.uint8)
    np.testing.assert_array_equal(digest, fx[f"{name}_occ_sha256"])


@pytest.mark.gpu
def test_rasterization_edge_cases():
    from dda_fft_b200 import Agglomerate, DDAGPUError
    occ, nd = Agglomerate.rasterize((16, 16, 16), np.zeros((0, 13), np.float32))
    assert nd == 0 and not occ.any()
    # one sphere monomer at the centre: every cell within its radius, none outside
    m = np.zeros((1, 13), np.float32)
    m[0, 0] = 3.0
    m[0, 8] = 1.0
    occ, nd = Agglomerate.rasterize((16, 32, 8), m)
    c = np.array([7.5, 15.5, 3.5], np.float32)
    idx = np.indices((16, 32, 8)).reshape(3, -1).T.astype(np.float32) - c
    d2 = (idx[:, 0] * idx[:, 0] + idx[:, 1] * idx[:, 1]) + idx[:, 2] * idx[:, 2]
    ref = (d2 <= 9.0) & (d2 <= 64.0)
    assert nd == int(ref.sum())
    np.testing.assert_array_equal(occ.ravel() != 0, ref)
    with pytest.raises(DDAGPUError):
        Agglomerate.rasterize((12, 16, 16), m)


# ---------------------------------------------------------------- random (Voronoi) ellipsoids
RELL = ["rell32", "rell64", "rell16"]


def rell_cfg(fx, name):
    ni, nj, nl, ba, ca, seed = fx[f"{name}_cfg"]
    return (int(ni), int(nj), int(nl)), float(ba), float(ca), int(seed)


@pytest.mark.parametrize("name", RELL)
def test_random_ellipsoid_seed_stream(fx, name):
    """The seed draws consume the reference's stream exactly (the next draw after them
    matches) and every seed lies on the lattice."""
    from dda_fft_b200 import RandomEllipsoid
    grid, ba, ca, seed = rell_cfg(fx, name)
    sps = fx[f"{name}_seeds_per_material"]
    r = RandomEllipsoid(state=seed)
    sd = r.seeds(grid, ba, ca, int(sps.sum()))
    assert next_draw(r.state) == int(fx[f"{name}_count_next"][1])
    assert (sd >= 0).all() and (sd <= np.array(grid) - 1).all()
    assert np.array_equal(sd, np.round(sd))


def test_random_ellipsoid_rejects_misfit():
    from dda_fft_b200 import DDAGPUError, RandomEllipsoid
    with pytest.raises(DDAGPUError):
        RandomEllipsoid(state=3).seeds((32, 16, 32), 1.0, 1.0, 4)


@pytest.mark.gpu
@pytest.mark.parametrize("name", RELL)
def test_random_ellipsoid_matches_reference(fx, name):
    from dda_fft_b200 import RandomEllipsoid
    grid, ba, ca, seed = rell_cfg(fx, name)
    sps = fx[f"{name}_seeds_per_material"]
    occ, count, _ = RandomEllipsoid(state=seed).generate(grid, ba, ca, sps)
    np.testing.assert_array_equal(occ, fx[f"{name}_occ"])
    assert count == int(fx[f"{name}_count_next"][0])


@pytest.mark.parametrize("n,r,lr,seed", [(32, 3.0, 0.0, 5), (32, 2.0, 1.5, 17), (64, 3.0, 0.0, 23),
                                         (64, 2.5, 2.0, 41), (32, 1.5, 3.0, 99)])
def test_placement_matches_live_reference(n, r, lr, seed):
    """The placement (grid-bucketed and vectorised crossing test) against the reference's
    own iGenerateAnthrax compiled from its sources, on seeds and shapes beyond the fixtures:
    the same monomers bit for bit and the same next draw."""
    import sys
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as P
    if not os.path.exists(P.REF_SO):
        pytest.skip("reference library not built")
    from dda_fft_b200 import Agglomerate
    count = Agglomerate.count((n, n, n), 0.25, r, lr)
    _, _, cyl, nxt = P.RefLib().gen_anthrax(seed, n, r, r * lr, count)
    a = Agglomerate(state=seed)
    mon = a.place(n, r, r * lr, count)
    np.testing.assert_array_equal(mon, cyl.astype(np.float32))
    assert next_draw(a.state) == nxt
