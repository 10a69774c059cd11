"""Solver iterations recorded as one CUDA graph (conditional while node) against the host
loop: same kernels in the same order, so the same discrepancy traces, steps and outputs
(up to the order of FP64 atomic additions), for every solver, single and batched."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def D():
    import dda_fft_b200
    return dda_fft_b200


def problem(oracle, n=16, x=4.0):
    occ, _ = oracle.gen_ellipsoid(n, n, n, 0.8, 0.6)
    kd = 2 * x / n
    m = complex(1.6, 0.002)
    a = kd ** 3 * (0.75 / np.pi) * (m * m - 1) / (m * m + 2)
    alpha = np.array([0, a], np.complex64)
    th = np.deg2rad(np.arange(19) * 10.0)
    ksc = np.stack([np.sin(th), np.zeros_like(th), np.cos(th)], 1)[None]
    return occ, kd, alpha, ksc


@pytest.mark.parametrize("solver", [0, 1, 2, 3])
def test_graph_equals_host_loop(D, oracle, solver):
    occ, kd, alpha, ksc = problem(oracle)
    tau = 0.6 if solver == 3 else 0.0
    out = {}
    with D.Context(occ.shape, kd) as ctx:
        for g in (False, True):
            ctx.set_solver_graph(g)
            runs0 = ctx.solver_graph_runs
            out[g] = ctx.dda_fft(occ, alpha, [0, 1], kd, (0, 0, 1), (1, 0, 0), ksc, solver=solver,
                                 tau=tau, max_step=40, err_max=1e-6)
            out[g, "runs"] = ctx.solver_graph_runs - runs0
    a, b = out[False], out[True]
    assert a["steps"] == b["steps"] and a["steps"] >= 2
    for q in ("step_min", "rolled_back", "matvecs"):
        assert a[q] == b[q], q
    assert out[True, "runs"] == 1 and out[False, "runs"] == 0
    n = a["steps"] + 1
    np.testing.assert_allclose(b["trace"][:n], a["trace"][:n], rtol=1e-9)
    for q in ("cext", "cabs"):
        assert abs(b[q] - a[q]) <= 1e-6 * abs(a[q])
    np.testing.assert_allclose(b["esc"], a["esc"], rtol=1e-5, atol=1e-7 * np.abs(a["esc"]).max())


def test_graph_batched_and_rebuilt(D, oracle):
    """Orientation batches with the graph: equal to the host loop; a different Max_Step
    rebuilds the graph and still stops where the host loop stops."""
    n, x = 16, 4.0
    occ, _ = oracle.gen_ellipsoid(n, n, n, 0.7, 0.5)
    rot = D.mc_rotations(7, 3)
    res = {}
    with D.Context(n, 2 * x / n, max_rhs=6) as ctx:
        for ms in (30, 7):
            for g in (False, True):
                ctx.set_solver_graph(g)
                cfg = D.BatchConfig(occ=occ, materials=[(1.6, 0.002)], err_max=1e-6, max_step=ms)
                res[ms, g] = ctx.orientation_solves(cfg, rot)
        assert ctx.solver_graph_runs == 2
    for ms in (30, 7):
        a, b = res[ms, False], res[ms, True]
        assert a["max_steps"] == b["max_steps"]
        np.testing.assert_allclose(b["cext"], a["cext"], rtol=1e-6)
        np.testing.assert_allclose(b["mueller"], a["mueller"], rtol=1e-5,
                                   atol=1e-7 * np.abs(a["mueller"]).max())
    assert res[7, True]["max_steps"] == 7


def test_graph_in_refinement(D, oracle):
    """Inner solves of the FP64-residual refinement run through the graph too."""
    occ, kd, alpha, ksc = problem(oracle)
    with D.Context(occ.shape, kd) as ctx:
        out = {}
        for g in (False, True):
            ctx.set_solver_graph(g)
            out[g] = ctx.dda_fft_refined(occ, alpha, [0, 1], kd, (0, 0, 1), (0, 1, 0), ksc,
                                         solver=2, err_max=1e-8, max_outer=20)
    assert out[True]["err"] <= 1e-8 and out[False]["err"] <= 1e-8
    assert abs(out[True]["cext"] - out[False]["cext"]) <= 1e-6 * abs(out[False]["cext"])


@pytest.mark.parametrize("max_step", [1, 2, 3])
@pytest.mark.parametrize("solver", [0, 2])
def test_graph_short_runs(D, oracle, solver, max_step):
    """Max_Step at the edges of the graph (1: no graph; 2: one pass; 3): the same stopping
    step, best iterate and rollback as the host loop."""
    occ, kd, alpha, ksc = problem(oracle)
    out = {}
    with D.Context(occ.shape, kd) as ctx:
        for g in (False, True):
            ctx.set_solver_graph(g)
            out[g] = ctx.dda_fft(occ, alpha, [0, 1], kd, (0, 0, 1), (1, 0, 0), ksc, solver=solver,
                                 max_step=max_step, err_max=1e-9)
    a, b = out[False], out[True]
    for q in ("steps", "step_min", "rolled_back", "matvecs"):
        assert a[q] == b[q], q
    assert a["steps"] == max_step
    np.testing.assert_allclose(b["trace"], a["trace"], rtol=1e-9)
    assert abs(b["cext"] - a["cext"]) <= 1e-6 * abs(a["cext"])


@pytest.mark.parametrize("xv", [3, 9])
def test_bounded_wait_reports_and_recovers(D, oracle, xv):
    """The x pass's bounded wait on its bulk copies (xv 3) and TMA tensor tiles (xv 9): a
    wait made to run out (self-test: after the copies have landed, a barrier phase nothing
    completes) fails the call with DDAGPU_ECUDA instead of hanging, and the context
    computes correctly again afterwards."""
    occ, kd, alpha, ksc = problem(oracle)
    rng = np.random.default_rng(2)
    p = (rng.standard_normal(occ.shape + (3,)) + 1j * rng.standard_normal(occ.shape + (3,))).astype(np.complex64)
    with D.Context(occ.shape, kd) as ctx:
        ctx.set_fast_variant(xv, 0)
        ref = ctx.convolution(p)
        ctx.selftest_wait_timeout(True)
        with pytest.raises(D.DDAGPUError, match="wait ran out"):
            ctx.convolution(p)
        with pytest.raises(D.DDAGPUError, match="wait ran out"):
            ctx.dda_fft(occ, alpha, [0, 1], kd, (0, 0, 1), (1, 0, 0), ksc, max_step=5)
        ctx.selftest_wait_timeout(False)
        again = ctx.convolution(p)
        np.testing.assert_array_equal(again, ref)
        r = ctx.dda_fft(occ, alpha, [0, 1], kd, (0, 0, 1), (1, 0, 0), ksc, max_step=5)
        assert r["steps"] >= 1
