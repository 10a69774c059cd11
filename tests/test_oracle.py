"""Pins the FP64 oracle (oracle/dda_oracle.c) to the reference's own outputs.

The golden fixtures come from the reference itself (tests/golden/make_golden.py): its
float build, its FP64 build (`typedef double real` + legacy FFT) and its unmodified
executable.  Against the FP64 build the oracle must agree to rounding (1e-10 relative);
against the float build to the float build's own noise.
"""
import numpy as np
import pytest

from pyoracle import orientation_solves


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("N", [8, 16, 32, 64, 128, 256])
def test_fft_line_known_answers(golden, oracle, N):
    """fft_bench.cpp's delta/roundtrip checks: both reference kernels vs the oracle DFT."""
    x = golden[f"fft{N}_in"]
    f = oracle.dft_line(x)
    b = oracle.dft_line(x, inverse=True)
    # the mixed-radix kernel uses FP64-built twiddles; the legacy radix-2 kernel a float
    # recurrence (fft_func.cpp:80-90), whose error grows with N (fft_bench.cpp gates 1e-5)
    assert rel(golden[f"fft{N}_fwd"], f) < 2e-6
    assert rel(golden[f"fft{N}_inv"], b) < 2e-6
    assert rel(golden[f"fft{N}_legacy_fwd"], f) < 1e-5
    assert rel(golden[f"fft{N}_legacy_inv"], b) < 1e-5
    # roundtrip FFT then iFFT = N x (fft_bench.cpp:394-430)
    assert rel(oracle.dft_line(f, inverse=True) / N, x) < 1e-12


def test_green_tensor(golden, oracle):
    n, kd = 8, float(golden["conv8_kd"])
    A = oracle.green_hat(n, n, n, kd)
    assert rel(A, golden["green8_hat64"]) < 1e-12
    assert rel(A, golden["green8_hat"]) < 2e-6


@pytest.mark.parametrize("n", [8, 16])
def test_convolution(golden, oracle, n):
    kd = float(golden[f"conv{n}_kd"])
    A = oracle.green_hat(n, n, n, kd)
    p = golden[f"conv{n}_p"].astype(np.complex128)
    out = oracle.convolution(A, p)
    assert rel(out, golden[f"conv{n}_out64"]) < 1e-12
    assert rel(out, golden[f"conv{n}_out"]) < 3e-6
    outc = oracle.convolution(A, p, conj=True)
    assert rel(outc, golden[f"conv{n}_out_conj"]) < 3e-6


def test_convolution_rectangular(golden, oracle):
    p = golden["convrect_p"].astype(np.complex128)
    A = oracle.green_hat(*p.shape[:3], float(golden["convrect_kd"]))
    assert rel(oracle.convolution(A, p), golden["convrect_out"]) < 3e-6


def test_symmetric_green_same_valid_block(golden, oracle):
    """Zeroing the index-n planes of G changes only discarded outputs."""
    n, kd = 8, float(golden["conv8_kd"])
    p = golden["conv8_p"].astype(np.complex128)
    a = oracle.convolution(oracle.green_hat(n, n, n, kd), p)
    b = oracle.convolution(oracle.green_hat(n, n, n, kd, zero_n_planes=True), p)
    assert rel(b, a) < 1e-13


@pytest.mark.parametrize("name", ["cg", "aa", "bicgstab", "simple", "simple_div"])
def test_solver_traces(golden, oracle, name):
    g = golden
    solver, tau, model, *einc = g[f"solve_{name}_cfg"]
    kd = float(g["solve_kd"])
    occ = g["solve_occ"]
    n = occ.shape[0]
    A = oracle.green_hat(n, n, n, kd)
    mv = np.array([0, 1])
    alpha = g[f"solve_{name}64_alpha"]
    r = oracle.dda_fft(occ, alpha, mv, kd, (0, 0, 1), einc, A, g["solve_ksc"].astype(np.float64),
                       solver=int(solver), tau=tau, max_step=8, err_max=1e-9)
    # the reference prints discrepancies with %9.7Lf
    assert np.abs(r["trace"] - g[f"solve_{name}64_trace"]).max() < 6e-8 * max(1, r["trace"].max())
    assert r["step_min"] == int(g[f"solve_{name}64_step_min"])
    assert rel(r["p"], g[f"solve_{name}64_p"]) < 1e-9
    assert rel(r["esc"], g[f"solve_{name}64_esc"]) < 1e-9
    assert abs(r["cabs"] - g[f"solve_{name}64_cabs"]) < 1e-9 * abs(r["cabs"])
    assert abs(r["cext"] - g[f"solve_{name}64_cext"]) < 1e-9 * abs(r["cext"])
    # and against the float build, within its own noise: the gate is
    # max(1e-4 relative, twice the float build's own distance from the FP64 build)
    for q in ("cext", "cabs"):
        ref32, ref64 = float(g[f"solve_{name}_{q}"]), float(g[f"solve_{name}64_{q}"])
        assert abs(r[q] - ref32) <= max(1e-4 * abs(ref32), 2 * abs(ref32 - ref64))


def test_jones_mueller(golden, oracle):
    e = golden["jm_e"]
    for k in range(len(e)):
        M = oracle.jones_mueller(golden["jm_kinc"][k], golden["jm_ksc"][k], golden["jm_nrm"][k],
                                 *e[k])[1]
        assert rel(M, golden["jm_mueller64"][k]) < 1e-12


def test_rng_and_geometry(golden, oracle):
    assert (oracle.rng(7, 64) == golden["rng_seed7"]).all()
    assert (oracle.rng(0, 16) == golden["rng_seed0"]).all()
    occ, n = oracle.gen_ellipsoid(16, 16, 16, 0.7, 0.5)
    assert (occ == golden["ellipsoid16_occ"]).all()


def test_polarizabilities(golden, oracle):
    for model, mre, mim, kd, are, aim in golden["pol_table"]:
        a = oracle.polarizability(int(model), kd, complex(mre, mim), (0, 0, 1), (0.6, 0.8, 0.0))
        assert abs(a - complex(are, aim)) < 1e-13 * abs(a)


def _dat_rows(golden):
    txt = bytes(golden["c1_dat"]).decode()
    lines = txt.strip().split("\n")
    head = lines[0].replace("\t", " ").split()
    ca, ce = float(head[0].split("=")[1]), float(head[1].split("=")[1])
    rows = np.array([[float(v) for v in ln.split()] for ln in lines[1:]])
    return ca, ce, rows


def test_config1_end_to_end(golden, oracle):
    """Config 1 (32^3 sphere, x=2, CG, 19 angles): oracle vs the reference executable."""
    ca, ce, rows = _dat_rows(golden)
    r = orientation_solves(oracle, 32, 2.0, [(1.5, 0.01)], 1)
    assert abs(r["cabs"] - ca) < 1e-4 * ca
    assert abs(r["cext"] - ce) < 3e-4 * ce   # float build vs FP64 noise at this config
    M = r["mueller"].reshape(-1, 16)
    scale = np.abs(rows[:, 1:]).max()
    sig = np.abs(rows[:, 1:]) > 1e-3 * scale
    err = np.abs(M - rows[:, 1:]) / np.maximum(np.abs(rows[:, 1:]), 1e-30)
    assert err[sig].max() < 1e-3


def test_monte_carlo_loop(golden, oracle):
    """MC orientations (seed 7, worker-0 stream) of a 16^3 ellipsoid vs the FP64 build."""
    ref = golden["mc16_n4_64"]
    r = orientation_solves(oracle, 16, 3.0, [(1.55, 0.005)], 4, target=2, b_a=0.7, c_a=0.5,
                           orientation=1, seed=7, nplanes=2)
    assert abs(r["cabs"] - ref[0]) < 1e-9 * abs(ref[0])
    assert abs(r["cext"] - ref[1]) < 1e-9 * abs(ref[1])
    assert rel(r["mueller"].ravel(), ref[2:]) < 1e-8


def test_ldr_bicgstab_loop(golden, oracle):
    ref = golden["ldr16_64"]
    r = orientation_solves(oracle, 16, 4.0, [(1.5, 0.01)], 1, polarizability=5, solver=2,
                           nplanes=3, theta_step=5.0, max_step=100)
    assert abs(r["cext"] - ref[1]) < 1e-9 * abs(ref[1])
    assert rel(r["mueller"].ravel(), ref[2:]) < 1e-8
