"""Generate the golden fixtures in tests/golden/ from the reference itself.

Every array here is an output of physicist2018/dda-fft's own code: the float build
(oracle/_ref/libddaref.so: the reference sources compiled where they lie, driven by
oracle/ref_shim.cpp), its FP64 build (oracle/_ref/libddaref64.so) and its unmodified
executable (oracle/_ref/dda_fft.out).  Run in a container that has the reference tree:

    make -f oracle/Makefile all && python tests/golden/make_golden.py
    python tests/golden/make_golden.py targets          # targets_v72.npz
    python tests/golden/make_golden.py configs          # configs_v72.npz (64^3, minutes)
    python tests/golden/make_golden.py fp64             # fp64_v72.npz (32^3 and 64^3 FP64 solves)

The fixtures are small (.npz, a few MB in all) and are committed; the tests read
them without needing the reference.
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
from pyoracle import REF64_SO, REF_EXE, RefLib, make_run_cfg  # noqa: E402


def cplx_rand(rng, shape, dt=np.complex64):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dt)


def fft_lines(R, out):
    rng = np.random.default_rng(101)
    for N in (8, 16, 32, 64, 128, 256):
        x = cplx_rand(rng, (N, 3))
        out[f"fft{N}_in"] = x
        for kind, name in ((0, "fwd"), (1, "inv"), (2, "legacy_fwd"), (3, "legacy_inv")):
            out[f"fft{N}_{name}"] = R.fft_line(x, kind)


def convolutions(R, R64, out):
    rng = np.random.default_rng(202)
    for n, x in ((8, 2.0), (16, 3.0)):
        kd = 2 * x / n
        A = R.green(n, n, n, kd)
        p = cplx_rand(rng, (n, n, n, 3))
        out[f"conv{n}_kd"] = kd
        out[f"conv{n}_p"] = p
        out[f"conv{n}_out"] = R.convolution(A, p)
        out[f"conv{n}_out_conj"] = R.convolution(A, p, conj=True)
        out[f"conv{n}_out64"] = R64.convolution(R64.green(n, n, n, kd), p.astype(np.complex128))
        if n == 8:
            out["green8_hat"] = A
            out["green8_hat64"] = R64.green(n, n, n, kd)
            out["green8_real"] = R.green_realspace(n, n, n, kd)
    # a non-cubic lattice (the reference's test matrix includes 32x64x32)
    n3 = (8, 16, 8)
    kd = 2 * 2.0 / n3[0]
    p = cplx_rand(rng, n3 + (3,))
    out["convrect_kd"] = kd
    out["convrect_p"] = p
    out["convrect_out"] = R.convolution(R.green(*n3, kd), p)


def solves(R, R64, out):
    """DDA_FFT traces for each solver on a 16^3 sphere (fixed orientation, 2 planes)."""
    n, x, m = 16, 3.0, 1.5 + 0.01j
    kd = 2 * x / n
    occ, nd = R.gen_ellipsoid(n, n, n)
    out["solve_occ"] = occ
    out["solve_kd"] = kd
    nP, nA = 2, 19
    # plane geometry as main.cpp:336-387 builds it (normal y, directions in xz), in float
    ksc = np.zeros((nP, nA, 3), np.float32)
    nrm = np.zeros((nP, 3), np.float32)
    for pl in range(nP):
        ang = np.float32(pl * 180.0 / nP) * (np.pi / 180.0)
        c, s = np.float32(np.cos(ang)), np.float32(np.sin(ang))
        nrm[pl] = (s, c, 0.0)
        for a in range(nA):
            th = np.float32(10.0 * a)
            k0 = np.array([np.sin(th * np.pi / 180), 0.0, np.cos(th * np.pi / 180)], np.float32)
            ksc[pl, a] = (c * k0[0] + s * k0[1], -s * k0[0] + c * k0[1], k0[2])
    out["solve_ksc"] = ksc
    out["solve_nrm"] = nrm
    A32 = R.green(n, n, n, kd)
    A64 = R64.green(n, n, n, kd)
    cases = [("cg", 0, 0.0, 1, (1, 0, 0)), ("aa", 1, 0.0, 2, (1, 0, 0)),
             ("bicgstab", 2, 0.0, 5, (0, 1, 0)), ("simple", 3, 0.5, 3, (1, 0, 0)),
             ("simple_div", 3, 3.0, 1, (1, 0, 0))]
    for name, solver, tau, model, einc in cases:
        a32 = R.polarizability(model, kd, m, (0, 0, 1), einc)
        a64 = R64.polarizability(model, kd, m, (0, 0, 1), einc)
        alpha32 = np.array([0, a32], np.complex64)
        alpha64 = np.array([0, a64], np.complex128)
        mv = np.array([0, 1], np.int32)
        for tag, L, A, al in (("", R, A32, alpha32), ("64", R64, A64, alpha64)):
            r = L.dda_fft(occ, al, mv, kd, (0, 0, 1), einc, A, ksc, solver=solver, tau=tau,
                          max_step=8, err_max=1e-9)
            out[f"solve_{name}{tag}_alpha"] = al
            out[f"solve_{name}{tag}_trace"] = r["trace"]
            out[f"solve_{name}{tag}_step_min"] = r["step_min"]
            out[f"solve_{name}{tag}_p"] = r["p"]
            out[f"solve_{name}{tag}_esc"] = r["esc"]
            out[f"solve_{name}{tag}_cabs"] = r["cabs"]
            out[f"solve_{name}{tag}_cext"] = r["cext"]
        out[f"solve_{name}_cfg"] = np.array([solver, tau, model] + list(einc), np.float64)


def jones(R, R64, out):
    rng = np.random.default_rng(303)
    K = 32
    ki = rng.standard_normal((K, 3))
    ki /= np.linalg.norm(ki, axis=1, keepdims=True)
    ks = rng.standard_normal((K, 3))
    ks /= np.linalg.norm(ks, axis=1, keepdims=True)
    nv = np.cross(ki, ks)
    nv /= np.linalg.norm(nv, axis=1, keepdims=True)
    e = cplx_rand(rng, (K, 4, 3), np.complex128)
    M = np.zeros((K, 4, 4))
    M32 = np.zeros((K, 4, 4), np.float32)
    for k in range(K):
        M[k] = R64.jones_mueller(ki[k], ks[k], nv[k], *e[k])[1]
        M32[k] = R.jones_mueller(ki[k], ks[k], nv[k], *e[k])[1]
    out.update(jm_kinc=ki, jm_ksc=ks, jm_nrm=nv, jm_e=e, jm_mueller64=M, jm_mueller=M32)


def misc(R, R64, out):
    out["rng_seed7"] = R.rng(7, 64)
    out["rng_seed0"] = R.rng(0, 16)
    pols = []
    for model in range(1, 6):
        for m in (1.5 + 0.01j, 1.7 + 0.1j, 1.33 + 0.0j):
            for kd in (0.125, 0.25, 0.5):
                pols.append((model, m.real, m.imag, kd, R64.polarizability(model, kd, m, (0, 0, 1),
                                                                        (0.6, 0.8, 0.0))))
    out["pol_table"] = np.array([(a, b, c, d, e.real, e.imag) for a, b, c, d, e in pols])
    occ, nd = R.gen_ellipsoid(16, 16, 16, 0.7, 0.5)
    out["ellipsoid16_occ"] = occ


def end_to_end(R, R64, out):
    """Config 1 through the unmodified executable, and MC sample loops through the shim."""
    cmd = [REF_EXE, "--target", "sphere", "--grid", "32", "-x", "2", "-m", "1.5", "0.01", "-P",
           "cm", "-M", "cg", "-e", "1e-3", "-S", "20", "--orientation", "fixed", "--planes", "1",
           "-a", "0", "-b", "180", "-s", "10", "--seed", "1", "--threads", "1", "--restart"]
    with tempfile.TemporaryDirectory() as td:
        subprocess.run(cmd + ["-o", "c1.dat", "-D", "c1.dst"], cwd=td, check=True,
                       capture_output=True)
        out["c1_dat"] = np.frombuffer(open(os.path.join(td, "c1.dat"), "rb").read(), np.uint8)
        out["c1_dst"] = np.frombuffer(open(os.path.join(td, "c1.dst"), "rb").read(), np.uint8)
    # the same configuration through the shim's sample loop (must equal the executable)
    cfg = make_run_cfg(grid=32, target=1, x=2.0, seed=1)
    s, ca, ce, mm = R.run_samples(cfg, 1, 1)
    out["c1_shim"] = np.concatenate([[ca, ce], mm.ravel()])
    # Monte-Carlo orientations of an ellipsoid, seed 7 (worker-0 stream), 16^3, x=3
    cfg = make_run_cfg(grid=16, target=2, b_a=0.7, c_a=0.5, x=3.0, materials=((1.55, 0.005),),
                       orientation=1, seed=7, nplanes=2, err_max=1e-3, max_step=20)
    for ns in (1, 4):
        s, ca, ce, mm = R.run_samples(cfg, ns, 1)
        out[f"mc16_n{ns}"] = np.concatenate([[ca, ce], mm.ravel()])
        s, ca, ce, mm = R64.run_samples(cfg, ns, 1)
        out[f"mc16_n{ns}_64"] = np.concatenate([[ca, ce], mm.ravel()])
    # LDR + BiCGStab + 3 planes at 16^3, x=4 (a small stand-in for the mid config)
    cfg = make_run_cfg(grid=16, target=1, x=4.0, polarizability=5, solver=2, nplanes=3,
                       theta_step=5.0, max_step=100, seed=1)
    s, ca, ce, mm = R.run_samples(cfg, 1, 1)
    out["ldr16"] = np.concatenate([[ca, ce], mm.ravel()])
    s, ca, ce, mm = R64.run_samples(cfg, 1, 1)
    out["ldr16_64"] = np.concatenate([[ca, ce], mm.ravel()])


# (name, lattice edge, monomer radius, length ratio, packing, generator seed): the
# agglomerate target of the realisation batch (radius 3, ratio 0, packing 0.25) and a
# capsule case with a cylindrical part
AGGLOMERATES = [("c3b32", 32, 3.0, 0.0, 0.25, 7), ("c3b64", 64, 3.0, 0.0, 0.25, 7),
                ("caps64", 64, 2.0, 2.5, 0.3, 99), ("c3b128", 128, 3.0, 0.0, 0.25, 7)]


# (name, lattice, b/a, c/a, seeds per material, generator seed)
RANDOM_ELLIPSOIDS = [("rell32", (32, 32, 32), 1.0, 1.0, [40], 5),
                     ("rell64", (64, 48, 32), 0.7, 0.5, [30, 20, 10], 9),
                     ("rell16", (16, 16, 16), 1.0, 1.0, [3, 0, 2], 1)]


def agglomerates(R, out):
    """iGenerateAnthrax (particle.cpp:21-85) after dda_srand(seed), monomer count as
    main.cpp:585-586: monomers, dipole count, the next draw of the stream, and the
    occupancy (bit-packed; as a SHA-256 only for 128^3)."""
    import hashlib
    for name, n, r, lr, rho, seed in AGGLOMERATES:
        count = int(rho * n ** 3 / (8.0 * r ** 3 * (0.75 * lr + 1))) + 1
        occ, nd, cyl, nxt = R.gen_anthrax(seed, n, r, r * lr, count)
        out[f"{name}_cfg"] = np.array([n, r, lr, rho, seed, count], np.float64)
        out[f"{name}_monomers"] = cyl.astype(np.float32)
        out[f"{name}_ndip_next"] = np.array([nd, nxt], np.int64)
        if n <= 64:
            out[f"{name}_occ_bits"] = np.packbits(occ.ravel() != 0)
        out[f"{name}_occ_sha256"] = np.frombuffer(
            hashlib.sha256((occ != 0).astype(np.uint8).tobytes()).digest(), np.uint8)
    # the reference's sample loop on agglomerates (one worker: realisations drawn one after
    # another from its stream), 32^3, x = 6, m = 1.55 + 0.005i, CM, CG, 3 samples
    cfg = make_run_cfg(grid=32, target=6, x=6.0, materials=((1.55, 0.005),), seed=7,
                       monomer_radius=3.0, monomer_ratio=0.0, packing=0.25)
    _, ca, ce, mm = R.run_samples(cfg, 3, 1)
    out["agg32_loop3"] = np.concatenate([[ca, ce], mm.ravel()])
    # random (Voronoi) ellipsoids, iGenerateRandomEllipsoid (particle.cpp:531-614)
    for name, grid, ba, ca_, sps, seed in RANDOM_ELLIPSOIDS:
        occ, n, nxt = R.gen_random_ellipsoid(seed, grid, ba, ca_, sps)
        out[f"{name}_cfg"] = np.array(list(grid) + [ba, ca_, seed], np.float64)
        out[f"{name}_seeds_per_material"] = np.array(sps, np.int32)
        out[f"{name}_occ"] = occ
        out[f"{name}_count_next"] = np.array([n, nxt], np.int64)


def full_configs(R, R64, out):
    """The mid and batching configurations at their full 64^3 size through the reference's
    sample loop (float and FP64 builds, one worker): sums of Cabs, Cext and the Mueller
    matrices, as the .dst holds them."""
    cfgs = {
        # 64^3 sphere, x = 8, m = 1.5+0.01i, LDR, BiCGStab, 100 steps, 12 planes, step 1 deg
        "c2": (make_run_cfg(grid=64, target=1, x=8.0, materials=((1.5, 0.01),), polarizability=5,
                            solver=2, max_step=100, nplanes=12, theta_step=1.0, seed=1), 1),
        # 64^3 ellipsoid 0.7/0.5, x = 6, m = 1.55+0.005i, CM, CG, MC orientations seed 7
        "c3a32": (make_run_cfg(grid=64, target=2, b_a=0.7, c_a=0.5, x=6.0,
                               materials=((1.55, 0.005),), orientation=1, seed=7), 32),
    }
    for name, (cfg, ns) in cfgs.items():
        _, ca, ce, mm = R.run_samples(cfg, ns, 1)
        out[name] = np.concatenate([[ca, ce], mm.ravel()])
        _, ca, ce, mm = R64.run_samples(cfg, ns, 1)
        out[name + "_64"] = np.concatenate([[ca, ce], mm.ravel()])
    # all 256 Monte-Carlo orientations of the batching configuration, one by one, in both
    # builds (worker 0's stream, as the single-threaded reference draws them)
    cfg = make_run_cfg(grid=64, target=2, b_a=0.7, c_a=0.5, x=6.0, materials=((1.55, 0.005),),
                       orientation=1, seed=7)
    for tag, L in (("", R), ("_64", R64)):
        _, _, _, _, (ca, ce, mm) = L.run_samples(cfg, 256, 1, each=True)
        out["c3a256_cabs" + tag] = ca
        out["c3a256_cext" + tag] = ce
        out["c3a256_mueller" + tag] = mm.reshape(256, -1, 16)


# FP64 solves of the reference's FP64 build at 32^3 and 64^3: (name, edge, x, m, solver,
# polarizability model, incident polarisation, steps).  Error_max is below reach, so every
# step runs; the fixtures keep the final dipoles of the middle plane i = n / 2.
FP64_SOLVES = [
    ("s32_bicg", 32, 4.0, 1.6 + 0.0005j, 2, 1, (1, 0, 0), 10),
    ("s32_cg", 32, 4.0, 1.6 + 0.0005j, 0, 2, (0, 1, 0), 16),
    ("s64_bicg", 64, 8.0, 1.5 + 0.01j, 2, 5, (1, 0, 0), 6),
    ("s64_cg", 64, 8.0, 1.6 + 0.0005j, 0, 1, (0, 1, 0), 10),
]


def fp64_solves(R64, out):
    """DDA_FFT of the reference's FP64 build on spheres at 32^3 and 64^3 (19 angles, one
    plane), for checking the GPU's FP64 solve."""
    th = np.deg2rad(np.arange(19) * 10.0)
    ksc = np.stack([np.sin(th), np.zeros_like(th), np.cos(th)], 1)[None]
    for name, n, x, m, solver, model, einc, steps in FP64_SOLVES:
        kd = 2 * x / n
        occ, _ = R64.gen_ellipsoid(n, n, n)
        a = R64.polarizability(model, kd, m, (0, 0, 1), einc)
        alpha = np.array([0, a], np.complex128)
        r = R64.dda_fft(occ, alpha, np.array([0, 1], np.int32), kd, (0, 0, 1), einc,
                        R64.green(n, n, n, kd), ksc, solver=solver, max_step=steps, err_max=1e-14)
        out[f"{name}_cfg"] = np.array([n, kd, solver, steps] + list(einc), np.float64)
        out[f"{name}_alpha"] = alpha
        out[f"{name}_trace"] = r["trace"]
        out[f"{name}_cext"] = r["cext"]
        out[f"{name}_cabs"] = r["cabs"]
        out[f"{name}_esc"] = r["esc"].reshape(-1, 3)
        out[f"{name}_pmid"] = r["p"][n // 2]
    out["fp64_ksc"] = ksc.reshape(-1, 3)


def main():
    if sys.argv[1:] == ["fp64"]:
        out: dict = {}
        fp64_solves(RefLib(REF64_SO), out)
        path = os.path.join(HERE, "fp64_v72.npz")
        np.savez_compressed(path, **out)
        print(f"wrote {path}: {os.path.getsize(path) / 1e6:.2f} MB, {len(out)} arrays")
        return
    if sys.argv[1:] == ["configs"]:
        out: dict = {}
        full_configs(RefLib(), RefLib(REF64_SO), out)
        path = os.path.join(HERE, "configs_v72.npz")
        np.savez_compressed(path, **out)
        print(f"wrote {path}: {os.path.getsize(path) / 1e6:.2f} MB, {len(out)} arrays")
        return
    if sys.argv[1:] == ["targets"]:
        out: dict = {}
        agglomerates(RefLib(), out)
        path = os.path.join(HERE, "targets_v72.npz")
        np.savez_compressed(path, **out)
        print(f"wrote {path}: {os.path.getsize(path) / 1e6:.2f} MB, {len(out)} arrays")
        return
    R = RefLib()
    R64 = RefLib(REF64_SO)
    assert R.rdt == np.float32 and R64.rdt == np.float64
    out: dict = {}
    fft_lines(R, out)
    convolutions(R, R64, out)
    solves(R, R64, out)
    jones(R, R64, out)
    misc(R, R64, out)
    end_to_end(R, R64, out)
    path = os.path.join(HERE, "reference_v72.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {os.path.getsize(path) / 1e6:.2f} MB, {len(out)} arrays")


if __name__ == "__main__":
    main()
