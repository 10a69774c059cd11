"""The mid and batching configurations at full size (64^3) against the reference's own
sample loop (float and FP64 builds; fixtures tests/golden/configs_v72.npz): sums of Cabs,
Cext and the plane-averaged Mueller matrices.  Gate: the float-noise gate of the other
parity tests, max(1e-4 |ref64|, 2 |ref32 - ref64|); significant Mueller elements to 1e-3
of the FP64 reference."""
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


def test_mid_configuration(D, oracle, fx):
    """64^3 sphere, x = 8, m = 1.5+0.01i, LDR, BiCGStab, 12 planes, 181 angles."""
    occ, _ = oracle.gen_ellipsoid(64, 64, 64, 1.0, 1.0)
    cfg = D.BatchConfig(occ=occ, materials=[(1.5, 0.01)], polarizability=5, solver=2,
                        max_step=100, nplanes=12, theta_step=1.0)
    with D.Context(64, 2 * 8.0 / 64, max_rhs=2) as ctx:
        r = ctx.orientation_solves(cfg, D.fixed_rotation(0, 0, 0)[None])
    assert r["mueller"].shape == (1, 181, 4, 4)
    check(r, fx["c2"], fx["c2_64"])


def test_batching_configuration_32_orientations(D, oracle, fx):
    """64^3 ellipsoid 0.7/0.5, x = 6, m = 1.55+0.005i, CM, CG, the first 32 Monte-Carlo
    orientations of seed 7, both polarisations, one batched call."""
    occ, _ = oracle.gen_ellipsoid(64, 64, 64, 0.7, 0.5)
    cfg = D.BatchConfig(occ=occ, materials=[(1.55, 0.005)])
    with D.Context(64, 2 * 6.0 / 64, max_rhs=64) as ctx:
        ctx.autotune(64)
        r = ctx.orientation_solves(cfg, D.mc_rotations(7, 32))
    check(r, fx["c3a32"], fx["c3a32_64"])
