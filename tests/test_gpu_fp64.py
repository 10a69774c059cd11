"""The FP64 GPU solve (ddagpu_solve_fp64) and the precision configuration pinned by it.

ddagpu_solve_fp64 is the reference's DDA_FFT with every field, transform, product and
scalar in double.  It is checked first against the reference's own FP64 build (golden
fixtures made by tests/golden/make_golden.py from oracle/_ref/libddaref64.so) at 16^3, 32^3
and 64^3 and against the FP64 C oracle on a rectangular lattice.  It then serves as the
independent FP64 solve of the 128^3 precision configuration, against which the FP32-matvec
refinement is measured: the refined answer is never its own reference.

The reference prints its per-step discrepancies with %9.7Lf (dda_func.cpp:1281,1525), so
the golden traces hold 7 decimals: they are compared to 6e-8 absolute.  Everything else is
compared to 1e-10 relative (both sides are FP64; the FFT algorithms and the Green tensor's
transform differ, so the last few digits do)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
TRACE_ABS = 6e-8      # the reference prints 7 decimals
FP64_REL = 1e-10


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="module")
def D():
    import dda_fft_b200
    return dda_fft_b200


@pytest.fixture(scope="module")
def fp64():
    return np.load(os.path.join(HERE, "golden", "fp64_v72.npz"))


@pytest.mark.parametrize("name", ["cg", "aa", "bicgstab", "simple", "simple_div"])
def test_fp64_solve_matches_reference_fp64_build_16(D, golden, name):
    """Every solver, 8 steps on a 16^3 sphere, against the reference's FP64 build."""
    g = golden
    cfg = g[f"solve_{name}_cfg"]
    solver, tau, einc = int(cfg[0]), float(cfg[1]), cfg[3:6]
    kd = float(g["solve_kd"])
    with D.Context(16, kd) as ctx:
        r = ctx.solve_fp64(g["solve_occ"], g[f"solve_{name}64_alpha"], [0, 1], kd, (0, 0, 1), einc,
                           g["solve_ksc"].astype(np.float64).reshape(-1, 3), solver=solver, tau=tau,
                           max_step=8, err_max=1e-9, want_p=True)
    tr = g[f"solve_{name}64_trace"]
    assert len(r["trace"]) == len(tr)
    assert np.abs(r["trace"] - tr).max() < TRACE_ABS
    assert r["step_min"] == int(g[f"solve_{name}64_step_min"])
    assert abs(r["cext"] - g[f"solve_{name}64_cext"]) < FP64_REL * abs(g[f"solve_{name}64_cext"])
    assert abs(r["cabs"] - g[f"solve_{name}64_cabs"]) < FP64_REL * abs(g[f"solve_{name}64_cabs"])
    assert rel(r["esc"], g[f"solve_{name}64_esc"].reshape(-1, 3)) < FP64_REL
    assert rel(r["p"], g[f"solve_{name}64_p"]) < FP64_REL


@pytest.mark.parametrize("name", ["s32_bicg", "s32_cg", "s64_bicg", "s64_cg"])
def test_fp64_solve_matches_reference_fp64_build(D, oracle, fp64, name):
    """Spheres at 32^3 and 64^3 (CM, CMRR, LDR; CG and BiCGStab), every step, against the
    reference's FP64 build: trace, cross sections, far field and the dipoles of the middle
    plane."""
    f = fp64
    n, kd, solver, steps = (int(f[f"{name}_cfg"][0]), float(f[f"{name}_cfg"][1]),
                            int(f[f"{name}_cfg"][2]), int(f[f"{name}_cfg"][3]))
    einc = f[f"{name}_cfg"][4:7]
    occ, _ = oracle.gen_ellipsoid(n, n, n)
    with D.Context(n, kd) as ctx:
        r = ctx.solve_fp64(occ, f[f"{name}_alpha"], [0, 1], kd, (0, 0, 1), einc, f["fp64_ksc"],
                           solver=solver, max_step=steps, err_max=1e-14, want_p=True)
    tr = f[f"{name}_trace"]
    assert len(r["trace"]) == len(tr) == steps + 1
    assert np.abs(r["trace"] - tr).max() < TRACE_ABS
    # BiCGStab's recurrence amplifies the last-digit differences of the two FFT algorithms
    # (measured: 2e-7 on Cext and 1.2e-6 on the dipoles after 10 steps at m = 1.6+0.0005i,
    # the traces still equal to the printed digits); CG keeps them at the last digits
    tol = FP64_REL if solver == 0 else 1e-5
    assert abs(r["cext"] - f[f"{name}_cext"]) < tol * abs(f[f"{name}_cext"])
    assert abs(r["cabs"] - f[f"{name}_cabs"]) < tol * abs(f[f"{name}_cabs"])
    assert rel(r["esc"], f[f"{name}_esc"]) < tol
    assert rel(r["p"][n // 2], f[f"{name}_pmid"]) < tol


@pytest.mark.parametrize("solver", [0, 1, 2, 3])
def test_fp64_solve_rectangular_and_rhs_vs_oracle(D, oracle, solver):
    """A rectangular lattice, a caller's right-hand side and a caller's starting field,
    against the FP64 C oracle's recurrences (no float casts)."""
    grid, kd = (8, 16, 4), 0.6
    rng = np.random.default_rng(solver)
    occ = (rng.random(grid) < 0.7).astype(np.int8) * rng.integers(1, 3, grid).astype(np.int8)
    alpha = np.array([0, oracle.polarizability(2, kd, 1.5 + 0.1j), oracle.polarizability(1, kd, 1.3 + 0.01j)])
    mv = [0, 1, 1]
    rhs = rng.standard_normal(grid + (3,)) + 1j * rng.standard_normal(grid + (3,))
    ksc = oracle.scattering_geometry(2, 7, 0.0, 30.0)[1]
    tau = 0.3 if solver == 3 else 0.0
    A = oracle.green_hat(*grid, kd)
    with D.Context(grid, kd) as ctx:
        r = ctx.solve_fp64(occ, alpha, mv, kd, (0, 0, 1), (1, 0, 0), ksc.reshape(-1, 3), solver=solver,
                           tau=tau, max_step=6, err_max=1e-14, rhs=rhs, want_p=True)
        x0 = r["p"]
        r2 = ctx.solve_fp64(occ, alpha, mv, kd, (0, 0, 1), (1, 0, 0), None, solver=0, max_step=3,
                            err_max=1e-14, rhs=rhs, x0=x0, want_p=True)
    o = oracle.dda_fft(occ, alpha, mv, kd, (0, 0, 1), (1, 0, 0), A, ksc, solver=solver, tau=tau,
                       max_step=6, err_max=1e-14, rhs=rhs)
    assert rel(r["trace"], o["trace"]) < 1e-9
    assert rel(r["p"], o["p"]) < 1e-9
    assert rel(r["esc"], o["esc"].reshape(-1, 3)) < 1e-9
    # started from the 6-step solution x0, the first discrepancy is that of A x0 - rhs: the
    # updated residual the first solve ended with (the simple iteration's residual belongs
    # to the iterate before its last update), and CG lowers it further
    if solver != 3:
        last = r["err_min"] if r["rolled_back"] else r["err"]
        assert r2["trace"][0] == pytest.approx(last, rel=1e-7)
    assert r2["trace"][1:].min() < r2["trace"][0]
