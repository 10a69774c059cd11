"""FP64-residual iterative refinement (precision pattern): FP32 inner solves through the
same matvec, FP64 solution and true residual.  Checked against FP64 oracle solves of the
same systems, at tolerances the float solvers alone cannot reach."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(oracle, n, x, m):
    kd = 2 * x / n
    occ, _ = oracle.gen_ellipsoid(n, n, n)
    alpha = np.array([0, oracle.polarizability(1, kd, m)])
    nrm, ksc = oracle.scattering_geometry(1, 46, 0.0, 4.0)
    return kd, occ, alpha, ksc


@pytest.mark.parametrize("n,x,solver", [(16, 4.0, 2), (16, 4.0, 0), (32, 5.0, 2)])
def test_refined_solve_matches_fp64_oracle(oracle, n, x, solver):
    import dda_fft_b200 as D
    m = 1.6 + 0.0005j                       # weakly absorbing: slow convergence
    kd, occ, alpha, ksc = _setup(oracle, n, x, m)
    with D.Context(n, kd) as ctx:
        r = ctx.dda_fft_refined(occ, alpha, [0, 1], kd, (0, 0, 1), (1, 0, 0), ksc, solver=solver,
                                err_max=1e-7, max_outer=30)
    assert r["err"] <= 1e-7, r["history"]
    o = oracle.dda_fft(occ, alpha, [0, 1], kd, (0, 0, 1), (1, 0, 0), oracle.green_hat(n, n, n, kd),
                       ksc, solver=solver, max_step=2000, err_max=1e-10)
    assert o["trace"][-1] <= 1e-10
    # the FP64 true residual makes the GPU solution agree with the converged FP64 one to
    # float-matvec accuracy, far below the float solver's own stagnation level
    assert abs(r["cext"] - o["cext"]) < 2e-5 * abs(o["cext"])
    assert abs(r["cabs"] - o["cabs"]) < 2e-5 * abs(o["cabs"])
    esc = r["esc"].reshape(-1, 3)
    oe = o["esc"].reshape(-1, 3)
    assert np.abs(esc - oe).max() < 2e-5 * np.abs(oe).max()


def test_refinement_reaches_below_float_stagnation(oracle):
    """A plain float BiCGStab run and the refined run on the same system: the refined true
    residual keeps decreasing geometrically."""
    import dda_fft_b200 as D
    n, x, m = 32, 6.0, 1.6 + 0.0005j
    kd, occ, alpha, ksc = _setup(oracle, n, x, m)
    with D.Context(n, kd) as ctx:
        r = ctx.dda_fft_refined(occ, alpha, [0, 1], kd, (0, 0, 1), (1, 0, 0), ksc, solver=2,
                                err_max=1e-8, max_outer=40, inner_rel=0.05, inner_max_step=300)
    h = r["history"]
    assert r["err"] <= 1e-8, h
    assert h[0] > 1e3 * r["err"]
