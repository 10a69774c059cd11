"""The mid and batching configurations at full size (64^3) against the reference's own
sample loop (float and FP64 builds; fixtures tests/golden/configs_v72.npz).

Batching configuration: all 256 Monte-Carlo orientations of seed 7, each orientation's
Cext, Cabs and plane-averaged Mueller matrix against the reference's FP64 build, at the
1e-4 relative bound of the batched mixed-precision target (Mueller elements: the
significant ones, above 1e-3 of that orientation's largest).  Mid configuration (one
sample): the same 1e-4 bound against the FP64 build."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def D():
    import dda_fft_b200
    return dda_fft_b200


@pytest.fixture(scope="module")
def fx():
    return np.load(os.path.join(ROOT, "tests", "golden", "configs_v72.npz"))


def check(r, ref32, ref64, mtol=1e-3):
    for k, q in ((0, "cabs"), (1, "cext")):
        got = float(np.sum(r[q]))
        gate = max(1e-4 * abs(ref64[k]), 2 * abs(ref32[k] - ref64[k]))
        assert abs(got - ref64[k]) <= gate, (q, got, ref32[k], ref64[k])
    M = r["mueller"].sum(axis=0).ravel()
    M64 = ref64[2:]
    sig = np.abs(M64) > 1e-3 * np.abs(M64).max()
    assert (np.abs(M[sig] - M64[sig]) / np.abs(M64[sig])).max() < mtol


def test_batching_configuration_256_orientations_each(D, oracle, fx):
    """64^3 ellipsoid 0.7/0.5, x = 6, m = 1.55+0.005i, CM, CG, Error_max 1e-3: the 256
    Monte-Carlo orientations of seed 7 (worker 0's stream), 64 per batched call, every
    orientation against the reference's FP64 build on its own."""
    occ, _ = oracle.gen_ellipsoid(64, 64, 64, 0.7, 0.5)
    cfg = D.BatchConfig(occ=occ, materials=[(1.55, 0.005)])
    with D.Context(64, 2 * 6.0 / 64, max_rhs=128) as ctx:
        ctx.autotune(128)
        r = ctx.orientation_solves(cfg, D.mc_rotations(7, 256))
    ca, ce = fx["c3a256_cabs_64"], fx["c3a256_cext_64"]
    M64 = fx["c3a256_mueller_64"]                                 # [256][19][16]
    M = r["mueller"].reshape(256, -1, 16)
    e_ca = np.abs(r["cabs"] - ca) / np.abs(ca)
    e_ce = np.abs(r["cext"] - ce) / np.abs(ce)
    sig = np.abs(M64) > 1e-3 * np.abs(M64).max(axis=(1, 2), keepdims=True)
    e_m = np.abs(M - M64)[sig] / np.abs(M64)[sig]
    # the float build against the FP64 one, for scale
    f_ca = np.abs(fx["c3a256_cabs"] - ca) / np.abs(ca)
    f_m = np.abs(fx["c3a256_mueller"] - M64)[sig] / np.abs(M64)[sig]
    print(f"256 orientations vs FP64: Cabs max {e_ca.max():.2e}, Cext max {e_ce.max():.2e}, "
          f"significant Mueller max {e_m.max():.2e} median {np.median(e_m):.2e} "
          f"({sig.sum()} values); float reference: Cabs max {f_ca.max():.2e}, Mueller max {f_m.max():.2e}")
    assert e_ca.max() < 1e-4 and e_ce.max() < 1e-4
    assert e_m.max() < 1e-4


def test_mid_configuration(D, oracle, fx):
    """64^3 sphere, x = 8, m = 1.5+0.01i, LDR, BiCGStab, 12 planes, 181 angles."""
    occ, _ = oracle.gen_ellipsoid(64, 64, 64, 1.0, 1.0)
    cfg = D.BatchConfig(occ=occ, materials=[(1.5, 0.01)], polarizability=5, solver=2,
                        max_step=100, nplanes=12, theta_step=1.0)
    with D.Context(64, 2 * 8.0 / 64, max_rhs=2) as ctx:
        r = ctx.orientation_solves(cfg, D.fixed_rotation(0, 0, 0)[None])
    assert r["mueller"].shape == (1, 181, 4, 4)
    check(r, fx["c2"], fx["c2_64"], mtol=1e-4)
    ref64 = fx["c2_64"]
    for k, q in ((0, "cabs"), (1, "cext")):
        assert abs(r[q][0] - ref64[k]) < 1e-4 * abs(ref64[k])


def test_batching_configuration_32_orientations(D, oracle, fx):
    """64^3 ellipsoid 0.7/0.5, x = 6, m = 1.55+0.005i, CM, CG, the first 32 Monte-Carlo
    orientations of seed 7, both polarisations, one batched call."""
    occ, _ = oracle.gen_ellipsoid(64, 64, 64, 0.7, 0.5)
    cfg = D.BatchConfig(occ=occ, materials=[(1.55, 0.005)])
    with D.Context(64, 2 * 6.0 / 64, max_rhs=64) as ctx:
        ctx.autotune(64)
        r = ctx.orientation_solves(cfg, D.mc_rotations(7, 32))
    check(r, fx["c3a32"], fx["c3a32_64"])
