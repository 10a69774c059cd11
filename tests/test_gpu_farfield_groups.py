"""The far field by kz groups (ddagpu_set_farfield_mode): directions that share their z
component share the z sum of the separable phase.  Both forms against the FP64 oracle's
per-direction sum (FarField, dda_func.cpp:1576-1625) and against each other, on cubic and
rectangular lattices, with holes, several materials and a material switched off; the
mid configuration's whole sample loop with either form."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max()


def crand(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


@pytest.fixture(scope="module")
def D():
    import dda_fft_b200
    return dda_fft_b200


@pytest.mark.parametrize("grid", [(16, 16, 16), (8, 16, 32), (32, 8, 16)])
def test_farfield_by_kz_groups_vs_oracle(D, oracle, grid):
    """12 scattering planes about z, 19 angles: 19 groups of 12 directions.  A random
    occupancy (a quarter holes, three materials); material 2 is switched off in the
    activity list but its cells hold dipoles: both forms skip them."""
    rng = np.random.default_rng(5)
    ni, nj, nl = grid
    kd = 0.4
    occ = rng.integers(0, 4, size=grid).astype(np.int8)
    mv = np.array([0, 1, 0, 1])
    p = crand(rng, (ni, nj, nl, 3))
    p[occ == 0] = 0
    nrm, ksc = oracle.scattering_geometry(12, 19, 0.0, 10.0)
    with D.Context(grid, kd) as ctx:
        out = {}
        for mode, kernels in ((1, 2), (2, 4)):
            ctx.set_farfield_mode(mode)
            n0 = ctx.kernel_launches
            out[mode] = ctx.farfield(occ, mv, kd, p, ksc)
            assert ctx.kernel_launches - n0 == kernels, mode
    ref = np.array([oracle.farfield(occ, mv, kd, p, k) for k in ksc.reshape(-1, 3)])
    e1, e2, e12 = rel(out[1], ref), rel(out[2], ref), rel(out[2], out[1])
    print(f"{grid}: direct {e1:.2e}, by kz groups {e2:.2e} vs the oracle; forms differ by {e12:.2e}")
    assert e1 < 1e-5 and e2 < 1e-5 and e12 < 1e-5


def test_farfield_mode_choice_and_arguments(D, oracle):
    """Default mode: the grouped form for 12 planes x 181 angles on a 64^3 sphere (one
    sum per distinct kz saves ~9/10 of the work), the direct form for one plane of 19
    angles (every direction its own kz)."""
    n, kd = 64, 2 * 8.0 / 64
    occ, _ = oracle.gen_ellipsoid(n, n, n)
    mv = np.array([0, 1])
    rng = np.random.default_rng(8)
    p = crand(rng, (n, n, n, 3))
    p[occ == 0] = 0
    _, many = oracle.scattering_geometry(12, 181, 0.0, 1.0)
    _, few = oracle.scattering_geometry(1, 19, 0.0, 10.0)
    with D.Context(n, kd) as ctx:
        for ksc, kernels in ((many, 4), (few, 2)):
            n0 = ctx.kernel_launches
            ctx.farfield(occ, mv, kd, p, ksc)
            assert ctx.kernel_launches - n0 == kernels
        for bad in (-1, 3):
            with pytest.raises(D.DDAGPUError):
                ctx.set_farfield_mode(bad)


def test_mid_configuration_both_forms(D, oracle):
    """64^3 sphere, x = 8, m = 1.5+0.01i, LDR, BiCGStab, 12 planes x 181 angles through the
    batched entry point: the grouped far field (default) and the direct one give the same
    cross sections and Mueller matrix to FP32 rounding."""
    occ, _ = oracle.gen_ellipsoid(64, 64, 64, 1.0, 1.0)
    cfg = D.BatchConfig(occ=occ, materials=[(1.5, 0.01)], polarizability=5, solver=2,
                        max_step=100, nplanes=12, theta_step=1.0)
    res = {}
    with D.Context(64, 2 * 8.0 / 64, max_rhs=2) as ctx:
        for mode in (1, 0):
            ctx.set_farfield_mode(mode)
            res[mode] = ctx.orientation_solves(cfg, D.fixed_rotation(0, 0, 0)[None])
    a, b = res[0], res[1]
    for q in ("cabs", "cext"):
        assert abs(a[q][0] - b[q][0]) <= 1e-6 * abs(b[q][0]), q
    M, M1 = a["mueller"][0].reshape(-1, 16), b["mueller"][0].reshape(-1, 16)
    sig = np.abs(M1) > 1e-3 * np.abs(M1).max()
    err = (np.abs(M - M1)[sig] / np.abs(M1)[sig]).max()
    print(f"mid configuration: grouped vs direct far field, significant Mueller max {err:.2e}")
    assert err < 1e-5
