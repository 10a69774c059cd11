"""ctypes bindings for the checkers -- TEST INFRASTRUCTURE ONLY.

* ``Oracle``  -- this repository's FP64 C restatement (oracle/dda_oracle.c).
* ``RefLib``  -- the reference's own sources compiled where they lie (oracle/ref_shim.cpp
  + physicist2018/dda-fft v7.2), float build ``libddaref.so`` or the FP64 build
  ``libddaref64.so``.

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs import this module.

Array conventions (numpy): a field is complex (ni, nj, nl, 3); the Green tensor is
complex (2ni, 2nj, 2nl, 6) in the component order e00, e01, e02, e11, e12, e22;
occupancy is int8 (ni, nj, nl).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libddaoracle.so")
REF_SO = os.path.join(HERE, "_ref", "libddaref.so")
REF64_SO = os.path.join(HERE, "_ref", "libddaref64.so")
REF_EXE = os.path.join(HERE, "_ref", "dda_fft.out")

_p = C.c_void_p
_i = C.c_int
_d = C.c_double


def build_oracle(quiet: bool = True) -> None:
    """Compile oracle/_build/libddaoracle.so (and oracle/_ref when the reference exists)."""
    out = subprocess.run(["make", "-f", os.path.join(HERE, "Makefile"), "all"],
                         capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


class Oracle:
    """FP64 restatement of the reference path (dda_oracle.c)."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build_oracle()
        self.lib = C.CDLL(path)
        L = self.lib
        L.or_green_hat.argtypes = [_i, _i, _i, _d, _i, _p]
        L.or_convolution.argtypes = [_i, _i, _i, _p, _p, _p, _i]
        L.or_dft_line.argtypes = [_i, _i, _p, _p]
        L.or_polarizability.argtypes = [_i, _d, _d, _d, _p, _p, _p]
        L.or_first_approximation.argtypes = [_i, _i, _i, _p, _p, _p, _d, _p, _p, _p]
        L.or_farfield.argtypes = [_i, _i, _i, _p, _p, _d, _p, _p, _p]
        L.or_cabscext.argtypes = [_i, _i, _i, _p, _p, _d, _p, _p, _p, _p, _p]
        L.or_jones_mueller.argtypes = [_p] * 9
        L.or_rng.argtypes = [C.c_ulonglong, _i, _p]
        L.or_mc_rotations.argtypes = [C.c_ulonglong, _i, _i, _p]
        L.or_gen_ellipsoid.argtypes = [_i, _i, _i, _d, _d, _p]
        L.or_scattering_geometry.argtypes = [_i, _i, _d, _d, _p, _p]
        L.or_dda_fft.argtypes = [_p, _p]

    def green_hat(self, ni, nj, nl, kd, zero_n_planes=False):
        out = np.zeros((2 * ni, 2 * nj, 2 * nl, 6), np.complex128)
        self.lib.or_green_hat(ni, nj, nl, kd, int(zero_n_planes), _ptr(out))
        return out

    def convolution(self, ahat, p, conj=False):
        ni, nj, nl = p.shape[:3]
        a = _c(ahat, np.complex128)
        x = _c(p, np.complex128)
        out = np.zeros_like(x)
        self.lib.or_convolution(ni, nj, nl, _ptr(a), _ptr(x), _ptr(out), int(conj))
        return out

    def dft_line(self, x, inverse=False):
        x = _c(x, np.complex128)
        out = np.zeros_like(x)
        self.lib.or_dft_line(x.shape[0], int(inverse), _ptr(x), _ptr(out))
        return out

    def polarizability(self, model, d0, m, kinc=(0, 0, 1), einc=(1, 0, 0)):
        k = _c(kinc, np.float64)
        e = _c(einc, np.complex128)
        out = np.zeros(2)
        self.lib.or_polarizability(model, d0, float(np.real(m)), float(np.imag(m)), _ptr(k),
                                   _ptr(e), _ptr(out))
        return complex(out[0], out[1])

    def first_approximation(self, occ, alpha, listmv, d0, kinc, einc):
        ni, nj, nl = occ.shape
        o = _c(occ, np.int8)
        a = _c(alpha, np.complex128)
        mv = _c(listmv, np.int32)
        k = _c(kinc, np.float64)
        e = _c(einc, np.complex128)
        p = np.zeros((ni, nj, nl, 3), np.complex128)
        self.lib.or_first_approximation(ni, nj, nl, _ptr(mv), _ptr(a), _ptr(o), d0, _ptr(k),
                                        _ptr(e), _ptr(p))
        return p

    def farfield(self, occ, listmv, d0, p, ksc):
        ni, nj, nl = occ.shape
        o = _c(occ, np.int8)
        mv = _c(listmv, np.int32)
        x = _c(p, np.complex128)
        k = _c(ksc, np.float64)
        out = np.zeros(3, np.complex128)
        self.lib.or_farfield(ni, nj, nl, _ptr(mv), _ptr(o), d0, _ptr(x), _ptr(k), _ptr(out))
        return out

    def cabscext(self, occ, alpha, d0, kinc, einc, p):
        ni, nj, nl = occ.shape
        o = _c(occ, np.int8)
        a = _c(alpha, np.complex128)
        k = _c(kinc, np.float64)
        e = _c(einc, np.complex128)
        x = _c(p, np.complex128)
        ca, ce = _d(), _d()
        self.lib.or_cabscext(ni, nj, nl, _ptr(a), _ptr(o), d0, _ptr(k), _ptr(e), _ptr(x),
                             C.byref(ca), C.byref(ce))
        return ca.value, ce.value

    def jones_mueller(self, kinc, ksc, normal, einc0, einc1, esc0, esc1):
        args = [_c(kinc, np.float64), _c(ksc, np.float64), _c(normal, np.float64),
                _c(einc0, np.complex128), _c(einc1, np.complex128), _c(esc0, np.complex128),
                _c(esc1, np.complex128)]
        j = np.zeros(4, np.complex128)
        m = np.zeros(16)
        self.lib.or_jones_mueller(*[_ptr(a) for a in args], _ptr(j), _ptr(m))
        return j.reshape(2, 2), m.reshape(4, 4)

    def rng(self, seed, count):
        out = np.zeros(count, np.int32)
        self.lib.or_rng(C.c_ulonglong(seed), count, _ptr(out))
        return out

    def mc_rotations(self, base_seed, worker, count):
        out = np.zeros((count, 3, 3))
        self.lib.or_mc_rotations(C.c_ulonglong(base_seed), worker, count, _ptr(out))
        return out

    def gen_ellipsoid(self, ni, nj, nl, b_a=1.0, c_a=1.0):
        occ = np.zeros((ni, nj, nl), np.int8)
        n = self.lib.or_gen_ellipsoid(ni, nj, nl, b_a, c_a, _ptr(occ))
        return occ, n

    def scattering_geometry(self, nplanes, nangles, theta_min, theta_step):
        nrm = np.zeros((nplanes, 3))
        ksc = np.zeros((nplanes, nangles, 3))
        self.lib.or_scattering_geometry(nplanes, nangles, theta_min, theta_step, _ptr(nrm),
                                        _ptr(ksc))
        return nrm, ksc

    def dda_fft(self, occ, alpha, listmv, d0, kinc, einc, ahat, ksc, solver=0, tau=0.0,
                max_step=20, err_max=1e-3, cast_scalars_float=False, rhs=None):
        """DDA_FFT for one polarisation; returns a dict with p, esc, cabs, cext, trace."""
        ni, nj, nl = occ.shape
        o = _c(occ, np.int8)
        a = _c(alpha, np.complex128)
        mv = _c(listmv, np.int32)
        A = _c(ahat, np.complex128)
        ks = _c(ksc, np.float64)
        npl, nang = ks.shape[:2]

        class In(C.Structure):
            _fields_ = [("ni", _i), ("nj", _i), ("nl", _i), ("solver", _i), ("tau", _d),
                        ("nmat", _i), ("alpha", _p), ("listmv", _p), ("occ", _p),
                        ("max_step", _i), ("err_max", _d), ("d0", _d), ("kinc", _d * 3),
                        ("einc", _d * 6), ("ahat", _p), ("nplanes", _i), ("nangles", _i),
                        ("ksc", _p), ("cast", _i), ("rhs", _p)]

        class Out(C.Structure):
            _fields_ = [("p", _p), ("esc", _p), ("cabs", _d), ("cext", _d), ("trace", _p),
                        ("ntrace", _i), ("step_min", _i), ("matvecs", _i)]

        e = np.asarray(einc, np.complex128)
        ein = (_d * 6)(*[v for z in e for v in (z.real, z.imag)])
        kin = (_d * 3)(*[float(v) for v in kinc])
        y = None if rhs is None else _c(rhs, np.complex128)
        si = In(ni, nj, nl, solver, tau, len(a) - 1, _ptr(a), _ptr(mv), _ptr(o), max_step,
                err_max, d0, kin, ein, _ptr(A), npl, nang, _ptr(ks), int(cast_scalars_float),
                None if y is None else _ptr(y))
        p = np.zeros((ni, nj, nl, 3), np.complex128)
        esc = np.zeros((npl, nang, 3), np.complex128)
        trace = np.zeros(max_step + 1)
        so = Out(_ptr(p), _ptr(esc), 0.0, 0.0, _ptr(trace), 0, -1, 0)
        rc = self.lib.or_dda_fft(C.byref(si), C.byref(so))
        if rc != 0:
            raise RuntimeError(f"or_dda_fft failed: {rc}")
        return dict(p=p, esc=esc, cabs=so.cabs, cext=so.cext, trace=trace[: so.ntrace],
                    step_min=so.step_min, matvecs=so.matvecs)


class RunCfg(C.Structure):
    """dref_run_cfg of ref_shim.cpp: one run of the reference's sample loop."""
    _fields_ = [("ni", _i), ("nj", _i), ("nl", _i), ("target", _i), ("b_a", _d), ("c_a", _d),
                ("x", _d), ("nmat", _i), ("m", _d * 32), ("polarizability", _i), ("solver", _i),
                ("tau", _d), ("err_max", _d), ("max_step", _i), ("fft_mode", _i),
                ("orientation", _i), ("psi", _d), ("iota", _d), ("kappa", _d), ("nplanes", _i),
                ("theta_min", _d), ("theta_max", _d), ("theta_step", _d),
                ("seed", C.c_ulonglong), ("monomer_radius", _d), ("monomer_ratio", _d),
                ("packing", _d)]


def make_run_cfg(grid=32, target=1, b_a=1.0, c_a=1.0, x=2.0, materials=((1.5, 0.01),),
                 polarizability=1, solver=0, tau=0.0, err_max=1e-3, max_step=20, fft_mode=0,
                 orientation=0, psi=0.0, iota=0.0, kappa=0.0, nplanes=1, theta_min=0.0,
                 theta_max=180.0, theta_step=10.0, seed=1, monomer_radius=0.0, monomer_ratio=0.0,
                 packing=0.0):
    g = grid if isinstance(grid, (tuple, list)) else (grid, grid, grid)
    m = (_d * 32)()
    for k, (re, im) in enumerate(materials):
        m[2 * k], m[2 * k + 1] = re, im
    return RunCfg(g[0], g[1], g[2], target, b_a, c_a, x, len(materials), m, polarizability,
                  solver, tau, err_max, max_step, fft_mode, orientation, psi, iota, kappa,
                  nplanes, theta_min, theta_max, theta_step, seed, monomer_radius, monomer_ratio,
                  packing)


class RefLib:
    """The reference's own functions (ref_shim.cpp over the reference sources)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path + " (build with `make -f oracle/Makefile ref`)")
        self.lib = C.CDLL(path)
        L = self.lib
        L.dref_sizeof_real.restype = _i
        self.rdt = np.float32 if L.dref_sizeof_real() == 4 else np.float64
        self.cdt = np.complex64 if self.rdt == np.float32 else np.complex128
        L.dref_green.argtypes = [_i, _i, _i, _d, _i, _p]
        L.dref_green_realspace.argtypes = [_i, _i, _i, _d, _p]
        L.dref_convolution.argtypes = [_i, _i, _i, _i, _i, _p, _p, _p]
        L.dref_dda_fft.argtypes = [_i, _i, _i, _i, _d, _i, _p, _p, _p, _i, _d, _d, _p, _p, _i,
                                   _p, _i, _i, _p, _p, _p, _p, _p, _p, _p, _p]
        L.dref_farfield.argtypes = [_i, _i, _i, _i, _p, _p, _d, _p, _p, _p]
        L.dref_cabscext.argtypes = [_i, _i, _i, _i, _p, _p, _d, _p, _p, _p, _p, _p]
        L.dref_jones_mueller.argtypes = [_p] * 9
        L.dref_polarizability.argtypes = [_i, _d, _d, _d, _p, _p, _p]
        L.dref_fft_line.argtypes = [_i, _i, _p, _p]
        L.dref_gen_ellipsoid.argtypes = [_i, _i, _i, _d, _d, _p]
        L.dref_rng.argtypes = [C.c_ulonglong, _i, _p]
        L.dref_gen_anthrax.argtypes = [C.c_ulonglong, _i, _i, _i, _d, _d, _i, _p, _p, _p]
        L.dref_gen_random_ellipsoid.argtypes = [C.c_ulonglong, _i, _i, _i, _d, _d, _i, _p, _p, _p]
        L.dref_run_samples.argtypes = [C.POINTER(RunCfg), _p, _i, _i, _i, _p, _p, _p, _p, _p]
        L.dref_set_per_sample.argtypes = [_p]

    def green(self, ni, nj, nl, kd, fft_mode=0):
        out = np.zeros((2 * ni, 2 * nj, 2 * nl, 6), self.cdt)
        self.lib.dref_green(ni, nj, nl, kd, fft_mode, _ptr(out))
        return out

    def green_realspace(self, ni, nj, nl, kd):
        out = np.zeros((2 * ni, 2 * nj, 2 * nl, 6), self.cdt)
        self.lib.dref_green_realspace(ni, nj, nl, kd, _ptr(out))
        return out

    def convolution(self, ahat, p, fft_mode=0, conj=False):
        ni, nj, nl = p.shape[:3]
        a = _c(ahat, self.cdt)
        x = _c(p, self.cdt)
        out = np.zeros_like(x)
        self.lib.dref_convolution(ni, nj, nl, fft_mode, int(conj), _ptr(a), _ptr(x), _ptr(out))
        return out

    def dda_fft(self, occ, alpha, listmv, d0, kinc, einc, ahat, ksc, solver=0, tau=0.0,
                max_step=20, err_max=1e-3, fft_mode=0):
        ni, nj, nl = occ.shape
        o = _c(occ, np.int8)
        a = _c(alpha, self.cdt)
        mv = _c(listmv, np.int32)
        A = _c(ahat, self.cdt)
        ks = _c(ksc, self.rdt)
        npl, nang = ks.shape[:2]
        k = _c(kinc, self.rdt)
        e = _c(einc, self.cdt)
        esc = np.zeros((npl, nang, 3), self.cdt)
        p = np.zeros((ni, nj, nl, 3), self.cdt)
        cabs = np.zeros(1, self.rdt)
        cext = np.zeros(1, self.rdt)
        trace = np.zeros(max_step + 1)
        nt = C.c_int(0)
        smin = C.c_int(-1)
        self.lib.dref_dda_fft(ni, nj, nl, solver, tau, len(a) - 1, _ptr(a), _ptr(mv), _ptr(o),
                              max_step, err_max, d0, _ptr(k), _ptr(e), fft_mode, _ptr(A), npl,
                              nang, _ptr(ks), _ptr(esc), _ptr(cabs), _ptr(cext), _ptr(p),
                              _ptr(trace), C.byref(nt), C.byref(smin))
        return dict(p=p, esc=esc, cabs=float(cabs[0]), cext=float(cext[0]),
                    trace=trace[: nt.value], step_min=smin.value)

    def farfield(self, occ, listmv, d0, p, ksc):
        ni, nj, nl = occ.shape
        o = _c(occ, np.int8)
        mv = _c(listmv, np.int32)
        x = _c(p, self.cdt)
        k = _c(ksc, self.rdt)
        out = np.zeros(3, self.cdt)
        self.lib.dref_farfield(ni, nj, nl, len(mv) - 1, _ptr(mv), _ptr(o), d0, _ptr(x), _ptr(k),
                               _ptr(out))
        return out

    def cabscext(self, occ, alpha, d0, kinc, einc, p):
        ni, nj, nl = occ.shape
        o = _c(occ, np.int8)
        a = _c(alpha, self.cdt)
        k = _c(kinc, self.rdt)
        e = _c(einc, self.cdt)
        x = _c(p, self.cdt)
        ca = np.zeros(1, self.rdt)
        ce = np.zeros(1, self.rdt)
        self.lib.dref_cabscext(ni, nj, nl, len(a) - 1, _ptr(a), _ptr(o), d0, _ptr(k), _ptr(e),
                               _ptr(x), _ptr(ca), _ptr(ce))
        return float(ca[0]), float(ce[0])

    def jones_mueller(self, kinc, ksc, normal, einc0, einc1, esc0, esc1):
        args = [_c(kinc, self.rdt), _c(ksc, self.rdt), _c(normal, self.rdt),
                _c(einc0, self.cdt), _c(einc1, self.cdt), _c(esc0, self.cdt), _c(esc1, self.cdt)]
        j = np.zeros(4, self.cdt)
        m = np.zeros(16, self.rdt)
        self.lib.dref_jones_mueller(*[_ptr(a) for a in args], _ptr(j), _ptr(m))
        return j.reshape(2, 2), m.reshape(4, 4)

    def polarizability(self, model, d0, m, kinc=(0, 0, 1), einc=(1, 0, 0)):
        k = _c(kinc, self.rdt)
        e = _c(einc, self.cdt)
        out = np.zeros(2, self.rdt)
        self.lib.dref_polarizability(model, d0, float(np.real(m)), float(np.imag(m)), _ptr(k),
                                     _ptr(e), _ptr(out))
        return complex(out[0], out[1])

    def fft_line(self, x, kind=0):
        x = _c(x, self.cdt)
        out = np.zeros_like(x)
        rc = self.lib.dref_fft_line(x.shape[0], kind, _ptr(x), _ptr(out))
        if rc != 0:
            raise ValueError("no plan")
        return out

    def gen_ellipsoid(self, ni, nj, nl, b_a=1.0, c_a=1.0):
        occ = np.zeros((ni, nj, nl), np.int8)
        n = self.lib.dref_gen_ellipsoid(ni, nj, nl, b_a, c_a, _ptr(occ))
        return occ, n

    def rng(self, seed, count):
        out = np.zeros(count, np.int32)
        self.lib.dref_rng(C.c_ulonglong(seed), count, _ptr(out))
        return out

    def gen_anthrax(self, seed, n, radius, length, count):
        """iGenerateAnthrax after dda_srand(seed): (occ, ndip, monomers[count][13], next draw)."""
        occ = np.zeros((n, n, n), np.int8)
        cyl = np.zeros((count, 13), self.rdt)
        nxt = C.c_int(0)
        nd = self.lib.dref_gen_anthrax(C.c_ulonglong(seed), n, n, n, radius, length, count,
                                       _ptr(occ), _ptr(cyl), C.byref(nxt))
        return occ, nd, cyl, nxt.value

    def gen_random_ellipsoid(self, seed, grid, b_a, c_a, seeds_per_sort):
        """iGenerateRandomEllipsoid after dda_srand(seed): (occ, count, next draw)."""
        ni, nj, nl = grid
        occ = np.zeros((ni, nj, nl), np.int8)
        sps = np.ascontiguousarray(seeds_per_sort, np.int32)
        nxt = C.c_int(0)
        n = self.lib.dref_gen_random_ellipsoid(C.c_ulonglong(seed), ni, nj, nl, b_a, c_a, len(sps),
                                               _ptr(sps), _ptr(occ), C.byref(nxt))
        return occ, n, nxt.value

    def run_samples(self, cfg: RunCfg, nsamples, nthreads=1, occ=None, verbose=0, each=False):
        """The reference's sample loop; returns (seconds, cabs_sum, cext_sum, mueller_sum),
        and with each=True also the per-sample (cabs, cext, mueller[angles][4][4])."""
        na = int(round((cfg.theta_max - cfg.theta_min) / cfg.theta_step + 1))
        mm = np.zeros((na + 2, 4, 4), self.rdt)
        ca = np.zeros(1, self.rdt)
        ce = np.zeros(1, self.rdt)
        secs = C.c_double(0)
        nout = C.c_int(0)
        o = _c(occ, np.int8) if occ is not None else np.zeros(1, np.int8)
        per = np.zeros(nsamples * (2 + 16 * (na + 2)), self.rdt) if each else None
        self.lib.dref_set_per_sample(_ptr(per) if each else None)
        self.lib.dref_run_samples(C.byref(cfg), _ptr(o), nthreads, nsamples, verbose,
                                  C.byref(secs), _ptr(ca), _ptr(ce), _ptr(mm), C.byref(nout))
        out = (secs.value, float(ca[0]), float(ce[0]), mm[: nout.value].copy())
        if not each:
            return out
        n = nout.value   # the C side writes rows of 2 + 16 n reals
        per = per[: nsamples * (2 + 16 * n)].reshape(nsamples, 2 + 16 * n)
        return out + ((per[:, 0].copy(), per[:, 1].copy(), per[:, 2:].reshape(nsamples, n, 4, 4)),)


def orientation_solves(O: Oracle, grid, x, materials, nsamples, target=1, b_a=1.0, c_a=1.0,
                       polarizability=1, solver=0, tau=0.0, err_max=1e-3, max_step=20,
                       orientation=0, psi=0.0, iota=0.0, kappa=0.0, nplanes=1, theta_min=0.0,
                       theta_max=180.0, theta_step=10.0, seed=1, occ=None, ahat=None):
    """The reference's sample loop (main.cpp:777-986, worker 0 only) over the FP64 oracle.

    Returns dict(cabs, cext, mueller) holding SUMS over samples, like the .dst state
    (main.cpp:961-981).  Used as the CPU 'port' baseline and as the end-to-end checker.
    """
    ni, nj, nl = (grid, grid, grid) if np.isscalar(grid) else tuple(grid)
    kd = 2.0 * x / ni
    na = int(round((theta_max - theta_min) / theta_step + 1.0))
    nrm0, ksc0 = O.scattering_geometry(nplanes, na, theta_min, theta_step)
    if ahat is None:
        ahat = O.green_hat(ni, nj, nl, kd)
    if occ is None:
        occ, _ = O.gen_ellipsoid(ni, nj, nl, 1.0 if target == 1 else b_a,
                                 1.0 if target == 1 else c_a)
    nmat = len(materials)
    mv = np.array([0] + [0 if (m[0] == 1.0 and m[1] == 0.0) else 1 for m in materials], np.int32)
    base_model = 4 if polarizability == 5 else polarizability
    alpha0 = np.array([0] + [O.polarizability(base_model, kd, complex(*m)) for m in materials])
    kinc0 = np.array([0.0, 0.0, 1.0])
    einc0 = np.array([[1, 0, 0], [0, 1, 0]], np.complex128)
    if orientation == 0:
        def rz(a):
            c, s = np.cos(a), np.sin(a)
            return np.array([[c, s, 0], [-s, c, 0], [0, 0, 1]])

        def ry(a):
            c, s = np.cos(a), np.sin(a)
            return np.array([[c, 0, -s], [0, 1, 0], [s, 0, c]])

        def rx(a):
            c, s = np.cos(a), np.sin(a)
            return np.array([[1, 0, 0], [0, c, s], [0, -s, c]])
        d = np.pi / 180
        T = rx(-kappa * d) @ ry(-iota * d) @ rz(-psi * d)   # main.cpp:516-541
        rots = [T] * nsamples
    else:
        rots = list(O.mc_rotations(seed, 0, nsamples))
    cabs = cext = 0.0
    mm_sum = np.zeros((na, 4, 4))
    for T in rots:
        kinc = T @ kinc0
        einc = [T @ e for e in einc0]
        ksc = ksc0 @ T.T
        nrm = nrm0 @ T.T
        esc = []
        sa = se = 0.0
        for q in range(2):
            alpha = alpha0.copy()
            if polarizability == 5:
                alpha[1:] = [O.polarizability(5, kd, complex(*m), kinc, einc[q]) for m in materials]
            r = O.dda_fft(occ, alpha, mv, kd, kinc, einc[q], ahat, ksc, solver=solver, tau=tau,
                          max_step=max_step, err_max=err_max)
            sa += 0.5 * r["cabs"]
            se += 0.5 * r["cext"]
            esc.append(r["esc"])
        for a in range(na):
            acc = np.zeros((4, 4))
            for pl in range(nplanes):
                acc += O.jones_mueller(kinc, ksc[pl, a], nrm[pl], einc[0], einc[1],
                                       esc[0][pl, a], esc[1][pl, a])[1]
            mm_sum[a] += acc / nplanes
        cabs += sa
        cext += se
    return dict(cabs=cabs, cext=cext, mueller=mm_sum, n=len(rots))
