"""ctypes mirror of include/ddagpu.h.

Host arrays use numpy in the reference's layouts: a field is complex64 (ni, nj, nl, 3)
(cvector), the Green tensor complex64 (2ni, 2nj, 2nl, 6) (cmatrix), the occupancy int8
(ni, nj, nl) (cAlpha).  Device entry points take torch CUDA tensors in the
structure-of-arrays layout (nrhs, 3, ni, nj, nl) complex64.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def library_path() -> str:
    return os.path.join(HERE, "lib", "libddagpu.so")


def build(force: bool = False) -> str:
    """Compile libddagpu.so for sm_100a with nvcc (dda_fft_b200/csrc/Makefile)."""
    path = library_path()
    args = ["make", "-C", os.path.join(HERE, "csrc"), "-j4"]
    if force:
        args.insert(1, "-B")
    out = subprocess.run(args, capture_output=True, text=True)
    if out.returncode != 0 or not os.path.exists(path):
        raise RuntimeError("libddagpu build failed:\n" + out.stdout[-4000:] + out.stderr[-4000:])
    return path


class DDAGPUError(RuntimeError):
    pass


_lib = None
_lock = threading.Lock()
_p, _i, _f, _d = C.c_void_p, C.c_int, C.c_float, C.c_double


class SolveInfo(C.Structure):
    _fields_ = [("steps", _i), ("step_min", _i), ("rolled_back", _i), ("matvecs", _i),
                ("err", _d), ("err_min", _d)]


class RefineInfo(C.Structure):
    _fields_ = [("outer", _i), ("inner_steps", _i), ("matvecs", _i), ("err", _d),
                ("err_history", _d * 64)]


class _BatchCfg(C.Structure):
    _fields_ = [("solver", _i), ("tau", _f), ("max_step", _i), ("err_max", _f),
                ("polarizability", _i), ("n_mat", _i), ("m", _p), ("occ", _p), ("nplanes", _i),
                ("theta_min", _f), ("theta_max", _f), ("theta_step", _f)]


class BatchInfo(C.Structure):
    _fields_ = [("n_rhs", _i), ("max_steps", _i), ("rolled_back", _i), ("max_err", _d)]


def lib():
    """Load libddagpu.so (building it first if it is absent); raises if that fails."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = library_path()
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.ddagpu_version.restype = C.c_char_p
        L.ddagpu_last_error.restype = C.c_char_p
        L.ddagpu_binary_version.argtypes = [_i, C.POINTER(_i)]
        L.ddagpu_create.argtypes = [C.POINTER(_p), _i, _i, _i, _i, _d, _i]
        L.ddagpu_destroy.argtypes = [_p]
        L.ddagpu_set_green.argtypes = [_p, _p]
        L.ddagpu_convolution.argtypes = [_p, _p, _p, _i]
        L.ddagpu_dda_fft.argtypes = [_p, _i, _i, _f, _i, _i, _i, _p, _p, _i, _p, _i, _f, _f, _p,
                                     _p, _i, _i, _i, _p, _p, _p, _p, C.POINTER(SolveInfo), _p]
        L.ddagpu_farfield.argtypes = [_p, _p, _i, _p, _f, _p, _i, _p, _p]
        L.ddagpu_solve_fp64.argtypes = [_p, _i, _d, _p, _p, _i, _p, _d, _p, _p, _p, _p, _i, _d,
                                        _i, _p, _p, C.POINTER(_d), C.POINTER(_d), _p,
                                        C.POINTER(SolveInfo), _p]
        L.ddagpu_release_fp64.argtypes = [_p]
        L.ddagpu_solve_linear.argtypes = [_p, _i, _f, _p, _p, _i, _p, _p, _d, _i, _i, _d, _i, _p,
                                          C.POINTER(RefineInfo)]
        L.ddagpu_dda_fft_refined.argtypes = [_p, _i, _f, _p, _p, _i, _p, _f, _p, _p, _d, _i, _d,
                                             _i, _i, _i, _p, _p, _p, _p, C.POINTER(RefineInfo)]
        L.ddagpu_cabscext.argtypes = [_p, _f, _p, _p, _p, _i, _p, _p, _p, _p]
        L.ddagpu_mueller.argtypes = [_p, _p, _p, _p, _i, _i, _p, _p, _p, _p, _p]
        L.ddagpu_orientation_solves.argtypes = [_p, C.POINTER(_BatchCfg), _i, _p, _p, _p, _p,
                                                C.POINTER(BatchInfo)]
        L.ddagpu_realization_solves.argtypes = [_p, C.POINTER(_BatchCfg), _i, _p, _p, _p, _p, _p,
                                                C.POINTER(BatchInfo)]
        L.ddagpu_agglomerate_solves.argtypes = [_p, C.POINTER(_BatchCfg), _i, _p, _p, _p, _p, _p,
                                                _p, _p, C.POINTER(BatchInfo)]
        L.ddagpu_state_read.argtypes = [C.c_char_p, _i, _i, C.POINTER(_i), C.POINTER(_f),
                                        C.POINTER(_f), _p]
        L.ddagpu_state_write.argtypes = [C.c_char_p, _i, _f, _f, _i, _p]
        L.ddagpu_state_accumulate.argtypes = [_i, _p, _p, _i, _p, C.POINTER(_i), C.POINTER(_f),
                                              C.POINTER(_f), _p]
        L.ddagpu_write_dat.argtypes = [C.c_char_p, _i, _f, _f, _i, _f, _f, _p]
        L.ddagpu_num_angles.argtypes = [_f, _f, _f]
        L.ddagpu_mc_rotations.argtypes = [C.c_ulonglong, _i, _i, _p]
        L.ddagpu_fixed_rotation.argtypes = [_d, _d, _d, _p]
        L.ddagpu_convolution_dev.argtypes = [_p, _p, _p, _i, _i]
        L.ddagpu_stream.argtypes = [_p]
        L.ddagpu_stream.restype = _p
        L.ddagpu_kernel_launches.argtypes = [_p]
        L.ddagpu_kernel_launches.restype = C.c_longlong
        L.ddagpu_set_tiling.argtypes = [_p, _i, _i]
        L.ddagpu_get_tiling.argtypes = [_p, C.POINTER(_i), C.POINTER(_i)]
        L.ddagpu_autotune.argtypes = [_p, _i]
        L.ddagpu_set_kernels.argtypes = [_p, _i]
        L.ddagpu_group_create.argtypes = [C.POINTER(_p), _p, _i]
        L.ddagpu_group_destroy.argtypes = [_p]
        L.ddagpu_group_graph_runs.argtypes = [_p]
        L.ddagpu_group_graph_runs.restype = C.c_longlong
        L.ddagpu_group_agglomerate_solves.argtypes = [_p, C.POINTER(_BatchCfg), _p, _p, _p, _p, _p, _p,
                                                      _p, _p, C.POINTER(BatchInfo)]
        L.ddagpu_farfield_noalloc.argtypes = [_i, _i, _i, _i, _f, _p, _p, _i, _p, _i, _p, _p, _p]
        L.ddagpu_get_kernels.argtypes = [_p]
        L.ddagpu_set_fast_variant.argtypes = [_p, _i, _i]
        L.ddagpu_set_farfield_mode.argtypes = [_p, _i]
        L.ddagpu_farfield_plan.argtypes = [_p, _i, _i, _i, _i, _i, _i, C.c_double, _i, _p, _p]
        L.ddagpu_get_fast_variant.argtypes = [_p, C.POINTER(_i), C.POINTER(_i)]
        L.ddagpu_set_solver_graph.argtypes = [_p, _i]
        L.ddagpu_selftest_wait_timeout.argtypes = [_p, _i]
        L.ddagpu_solver_graph_runs.argtypes = [_p]
        L.ddagpu_solver_graph_runs.restype = C.c_longlong
        L.ddagpu_rng_seed.argtypes = [C.c_ulonglong, _i]
        L.ddagpu_rng_seed.restype = C.c_ulonglong
        L.ddagpu_anthrax_count.argtypes = [_i, _i, _i, _f, _f, _f]
        L.ddagpu_anthrax_count.restype = C.c_longlong
        L.ddagpu_anthrax_place.argtypes = [C.POINTER(C.c_ulonglong), _i, _f, _f, _i, _p]
        L.ddagpu_anthrax_rasterize.argtypes = [_i, _i, _i, _i, _p, _i, _p, C.POINTER(_i)]
        L.ddagpu_random_ellipsoid_seeds.argtypes = [C.POINTER(C.c_ulonglong), _i, _i, _i, _f, _f,
                                                    _i, _p]
        L.ddagpu_random_ellipsoid_fill.argtypes = [_i, _i, _i, _i, _f, _f, _p, _p, _i, _p,
                                                   C.POINTER(_i)]
        _lib = L
        return L


def _check(rc: int) -> None:
    if rc != 0:
        msg = lib().ddagpu_last_error().decode(errors="replace")
        raise DDAGPUError(f"libddagpu error {rc}: {msg}")


def _ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def _cvec(a):
    """complex (..., 3) -> float32 interleaved cvector layout."""
    return np.ascontiguousarray(np.asarray(a, np.complex64)).view(np.float32)


def num_angles(theta_min, theta_max, theta_step) -> int:
    return int(lib().ddagpu_num_angles(theta_min, theta_max, theta_step))


def mc_rotations(base_seed: int, count: int, worker: int = 0) -> np.ndarray:
    out = np.zeros((count, 3, 3))
    _check(lib().ddagpu_mc_rotations(C.c_ulonglong(base_seed), worker, count, _ptr(out)))
    return out


def farfield_plan(ksc, grid, nact: float, nrhs: int = 1, pairs: bool = False, mode: int = 0):
    """(groups, items) of the far field over the directions ksc of nrhs right-hand sides
    (any shape of nrhs x ndir x 3 values) on a lattice `grid` with `nact` active cells per
    right-hand side: groups 0 means one sum per direction (ddagpu_farfield_plan; no device
    needed)."""
    k = np.ascontiguousarray(ksc, np.float64).reshape(nrhs, -1, 3)
    ni, nj, nl = (grid,) * 3 if np.isscalar(grid) else grid
    g, it = C.c_int(), C.c_int()
    _check(lib().ddagpu_farfield_plan(_ptr(k), k.shape[0], k.shape[1], int(pairs), ni, nj, nl,
                                      float(nact), mode, C.byref(g), C.byref(it)))
    return g.value, it.value


def fixed_rotation(psi=0.0, iota=0.0, kappa=0.0) -> np.ndarray:
    out = np.zeros((3, 3))
    _check(lib().ddagpu_fixed_rotation(psi, iota, kappa, _ptr(out)))
    return out


class Agglomerate:
    """Anthrax-like agglomerates of capsule monomers (target 6, iGenerateAnthrax,
    particle.cpp:21-85): monomers placed on the host from the reference's random stream,
    rasterised into the lattice on the GPU.  `state` follows the stream across samples
    like the worker's generator does (main.cpp:803-830)."""

    def __init__(self, base_seed: int = 0, worker: int = 0, state: int | None = None):
        self.state = int(lib().ddagpu_rng_seed(C.c_ulonglong(base_seed), worker)
                         if state is None else state)

    @staticmethod
    def count(grid, packing: float, monomer_radius: float, length_ratio: float) -> int:
        ni, nj, nl = grid
        return int(lib().ddagpu_anthrax_count(ni, nj, nl, packing, monomer_radius, length_ratio))

    def place(self, i_max: int, monomer_radius: float, monomer_length: float,
              count: int) -> np.ndarray:
        """monomers[count][13] float32: r, l, begin xyz, end xyz, axis xyz, 0, 0."""
        out = np.zeros((count, 13), np.float32)
        s = C.c_ulonglong(self.state)
        _check(lib().ddagpu_anthrax_place(C.byref(s), i_max, monomer_radius, monomer_length,
                                          count, _ptr(out)))
        self.state = s.value
        return out

    @staticmethod
    def rasterize(grid, monomers: np.ndarray, device: int = 0):
        """(occ int8 [ni][nj][nl], 1 = filled; number of filled cells)."""
        ni, nj, nl = grid
        m = _f32(monomers)
        occ = np.zeros((ni, nj, nl), np.int8)
        nd = C.c_int(0)
        _check(lib().ddagpu_anthrax_rasterize(device, ni, nj, nl, _ptr(m), len(m), _ptr(occ),
                                              C.byref(nd)))
        return occ, nd.value

    def generate(self, grid, monomer_radius: float, monomer_length: float, count: int,
                 device: int = 0):
        mon = self.place(grid[0], monomer_radius, monomer_length, count)
        occ, nd = self.rasterize(grid, mon, device)
        return occ, nd, mon


class RandomEllipsoid:
    """Random (Voronoi) ellipsoids (targets 4 and 5, iGenerateRandomEllipsoid,
    particle.cpp:531-614): seeds drawn on the host from the reference's random stream,
    nearest-seed fill on the GPU; seeds_per_material[m] seeds give material m + 1."""

    def __init__(self, base_seed: int = 0, worker: int = 0, state: int | None = None):
        self.state = int(lib().ddagpu_rng_seed(C.c_ulonglong(base_seed), worker)
                         if state is None else state)

    def seeds(self, grid, b_a: float, c_a: float, n_seeds: int) -> np.ndarray:
        ni, nj, nl = grid
        out = np.zeros((n_seeds, 3), np.float32)
        s = C.c_ulonglong(self.state)
        _check(lib().ddagpu_random_ellipsoid_seeds(C.byref(s), ni, nj, nl, b_a, c_a, n_seeds,
                                                   _ptr(out)))
        self.state = s.value
        return out

    @staticmethod
    def fill(grid, b_a: float, c_a: float, seeds: np.ndarray, seeds_per_material,
             device: int = 0):
        """(occ int8 [ni][nj][nl] of materials 0..n_mat, the reference's count of
        material-1 cells)."""
        ni, nj, nl = grid
        sd = _f32(seeds)
        spm = np.ascontiguousarray(seeds_per_material, np.int32)
        occ = np.zeros((ni, nj, nl), np.int8)
        nd = C.c_int(0)
        _check(lib().ddagpu_random_ellipsoid_fill(device, ni, nj, nl, b_a, c_a, _ptr(sd),
                                                  _ptr(spm), len(spm), _ptr(occ), C.byref(nd)))
        return occ, nd.value

    def generate(self, grid, b_a: float, c_a: float, seeds_per_material, device: int = 0):
        sd = self.seeds(grid, b_a, c_a, int(np.sum(seeds_per_material)))
        occ, nd = self.fill(grid, b_a, c_a, sd, seeds_per_material, device)
        return occ, nd, sd


class StateFile:
    """The sample loop's .dst state in the reference's float layout (main.cpp:214-274,
    961-981): sample counter, float sums of Cabs, Cext and the Mueller matrices."""

    def __init__(self, path: str, n_angles: int, restart: bool = False):
        self.path, self.n_angles = os.fspath(path), int(n_angles)
        self.mueller = np.zeros((self.n_angles, 4, 4), np.float32)
        c, a, e = _i(0), _f(0), _f(0)
        _check(lib().ddagpu_state_read(self.path.encode(), self.n_angles, int(restart), C.byref(c),
                                       C.byref(a), C.byref(e), _ptr(self.mueller)))
        self.counter, self.cabs, self.cext = c.value, a.value, e.value

    def add(self, result: dict) -> None:
        """Accumulate the samples of one batched call (orientation_solves,
        realization_solves, agglomerate_solves), in order."""
        ca = np.ascontiguousarray(result["cabs"], np.float64)
        ce = np.ascontiguousarray(result["cext"], np.float64)
        mm = np.ascontiguousarray(result["mueller"], np.float64)
        c, a, e = _i(self.counter), _f(self.cabs), _f(self.cext)
        _check(lib().ddagpu_state_accumulate(len(ca), _ptr(ca), _ptr(ce), self.n_angles, _ptr(mm),
                                             C.byref(c), C.byref(a), C.byref(e),
                                             _ptr(self.mueller)))
        self.counter, self.cabs, self.cext = c.value, a.value, e.value

    def save(self) -> None:
        _check(lib().ddagpu_state_write(self.path.encode(), self.counter, self.cabs, self.cext,
                                        self.n_angles, _ptr(self.mueller)))

    def write_dat(self, path: str, theta_min: float = 0.0, theta_step: float = 10.0) -> None:
        """The .dat of main.cpp:1085-1118 (averages over the counter)."""
        _check(lib().ddagpu_write_dat(os.fspath(path).encode(), self.counter, self.cabs, self.cext,
                                      self.n_angles, theta_min, theta_step, _ptr(self.mueller)))


def sample_loop(ctx, cfg, samples: int, state_path: str, dat_path: str | None = None,
                orientation: str = "fixed", seed: int = 1, psi: float = 0.0, iota: float = 0.0,
                kappa: float = 0.0, restart: bool = False, batch: int | None = None):
    """The reference's sample loop for one worker (main.cpp:214-320, 689-986, 1085-1118)
    over the batched GPU solves: open or create the state, solve the samples still missing
    (samples - counter) in batches, refresh the state after every batch and write the .dat.
    Like the reference, a resumed run numbers its samples after the stored ones but
    restarts the worker's random stream (main.cpp:803-804), so its Monte-Carlo draws
    repeat those of the first run."""
    na = num_angles(cfg.theta_min, cfg.theta_max, cfg.theta_step)
    st = StateFile(state_path, na, restart)
    tasks = max(samples - st.counter, 0)
    if orientation == "mc":
        rot = mc_rotations(seed, tasks) if tasks else np.zeros((0, 3, 3))
    elif orientation == "fixed":
        rot = np.repeat(fixed_rotation(psi, iota, kappa)[None], tasks, axis=0)
    else:
        raise ValueError("orientation must be 'fixed' or 'mc'")
    per = batch or max(ctx.max_rhs // 2, 1)
    first = True
    for s0 in range(0, tasks, per):
        c = cfg if first else BatchConfig(**{**cfg.__dict__, "occ": None})
        st.add(ctx.orientation_solves(c, rot[s0:s0 + per]))
        st.save()
        first = False
    if dat_path is not None and st.counter > 0:
        st.write_dat(dat_path, cfg.theta_min, cfg.theta_step)
    return st


@dataclass
class BatchConfig:
    occ: np.ndarray | None     # None: reuse the occupancy resident from the previous call
    materials: list = field(default_factory=lambda: [(1.5, 0.01)])
    solver: int = 0
    tau: float = 0.0
    max_step: int = 20
    err_max: float = 1e-3
    polarizability: int = 1
    nplanes: int = 1
    theta_min: float = 0.0
    theta_max: float = 180.0
    theta_step: float = 10.0


class Context:
    """One lattice on one GPU (ddagpu_create)."""

    def __init__(self, grid, kd: float, max_rhs: int = 1, device: int = 0):
        self.grid = (grid,) * 3 if np.isscalar(grid) else tuple(int(g) for g in grid)
        self.kd = float(kd)
        self.max_rhs = max_rhs
        h = C.c_void_p()
        _check(lib().ddagpu_create(C.byref(h), device, *self.grid, self.kd, max_rhs))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().ddagpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    @property
    def kernel_launches(self) -> int:
        return int(lib().ddagpu_kernel_launches(self._h))

    @property
    def stream_ptr(self) -> int:
        return int(lib().ddagpu_stream(self._h) or 0)

    def set_green(self, cmA: np.ndarray) -> None:
        a = np.ascontiguousarray(np.asarray(cmA, np.complex64))
        _check(lib().ddagpu_set_green(self._h, _ptr(a)))

    def convolution(self, p: np.ndarray, conj: bool = False) -> np.ndarray:
        x = _cvec(p)
        out = np.zeros_like(x)
        _check(lib().ddagpu_convolution(self._h, _ptr(x), _ptr(out), int(conj)))
        return out.view(np.complex64).reshape(np.shape(p))

    def dda_fft(self, occ, alpha, listmv, d0, kinc, einc, ksc, solver=0, tau=0.0, max_step=20,
                err_max=1e-3, fft_mode=0, trace=True):
        """DDA_FFT for one polarisation; returns dict(esc, cabs, cext, info, trace)."""
        o = np.ascontiguousarray(occ, np.int8)
        a = _cvec(np.asarray(alpha, np.complex64).reshape(-1, 1)).ravel()
        mv = np.ascontiguousarray(listmv, np.int32)
        ks = _f32(ksc)
        npl, nang = ks.shape[:2]
        esc = np.zeros((npl, nang, 3), np.complex64)
        k = _f32(kinc)
        e = _cvec(np.asarray(einc, np.complex64))
        ca, ce = C.c_float(), C.c_float()
        info = SolveInfo()
        tr = np.zeros(max_step + 1) if trace else None
        _check(lib().ddagpu_dda_fft(self._h, 0, solver, tau, *self.grid, _ptr(a), _ptr(mv),
                                    len(mv) - 1, _ptr(o), max_step, err_max, d0, _ptr(k), _ptr(e),
                                    fft_mode, npl, nang, _ptr(ks), _ptr(esc.view(np.float32)),
                                    C.byref(ca), C.byref(ce), C.byref(info),
                                    _ptr(tr) if trace else None))
        out = dict(esc=esc, cabs=ca.value, cext=ce.value, steps=info.steps,
                   step_min=info.step_min if info.rolled_back else -1, matvecs=info.matvecs,
                   err=info.err, err_min=info.err_min, rolled_back=info.rolled_back)
        if trace:
            out["trace"] = tr[: info.steps + 1]
        return out

    def dda_fft_refined(self, occ, alpha, listmv, d0, kinc, einc, ksc, solver=2, tau=0.0,
                        err_max=1e-5, max_outer=20, inner_rel=None, inner_max_step=None):
        """FP64-residual iterative refinement around the chosen solver.  CG (solver 0) runs
        with FP64 fields and scalars between true residuals (defaults: inner_rel 1e-3,
        inner_max_step 5000); the other solvers run in FP32 (defaults 0.05, 200)."""
        if inner_rel is None:
            inner_rel = 1e-3 if solver == 0 else 0.05
        if inner_max_step is None:
            inner_max_step = 5000 if solver == 0 else 200
        o = np.ascontiguousarray(occ, np.int8)
        a = _cvec(np.asarray(alpha, np.complex64).reshape(-1, 1)).ravel()
        mv = np.ascontiguousarray(listmv, np.int32)
        ks = _f32(ksc)
        npl, nang = ks.shape[:2]
        esc = np.zeros((npl, nang, 3), np.complex64)
        k = _f32(kinc)
        e = _cvec(np.asarray(einc, np.complex64))
        ca, ce = C.c_float(), C.c_float()
        info = RefineInfo()
        _check(lib().ddagpu_dda_fft_refined(self._h, solver, tau, _ptr(a), _ptr(mv), len(mv) - 1,
                                            _ptr(o), d0, _ptr(k), _ptr(e), err_max, max_outer,
                                            inner_rel, inner_max_step, npl, nang, _ptr(ks),
                                            _ptr(esc.view(np.float32)), C.byref(ca), C.byref(ce),
                                            C.byref(info)))
        hist = np.array(info.err_history[: min(info.outer + 1, 64)])
        return dict(esc=esc, cabs=ca.value, cext=ce.value, outer=info.outer,
                    inner_steps=info.inner_steps, matvecs=info.matvecs, err=info.err, history=hist)

    def solve_linear(self, occ, alpha, listmv, rhs, solver=0, tau=0.0, err_max=1e-8,
                     max_step=40, refine=True, inner_rel=None, inner_max_step=None):
        """x with (I - D_alpha G) x = rhs; rhs complex (ni, nj, nl, 3).  inner_rel and
        inner_max_step as for dda_fft_refined."""
        if inner_rel is None:
            inner_rel = 1e-3 if solver == 0 else 0.05
        if inner_max_step is None:
            inner_max_step = 5000 if solver == 0 else 300
        o = np.ascontiguousarray(occ, np.int8)
        a = _cvec(np.asarray(alpha, np.complex64).reshape(-1, 1)).ravel()
        mv = np.ascontiguousarray(listmv, np.int32)
        b = _cvec(rhs)
        x = np.zeros_like(b)
        info = RefineInfo()
        _check(lib().ddagpu_solve_linear(self._h, solver, tau, _ptr(a), _ptr(mv), len(mv) - 1,
                                         _ptr(o), _ptr(b), err_max, max_step, int(refine),
                                         inner_rel, inner_max_step, _ptr(x), C.byref(info)))
        hist = np.array(info.err_history[: min(info.outer + 1, 64)])
        return x.view(np.complex64).reshape(np.shape(rhs)), dict(
            outer=info.outer, inner_steps=info.inner_steps, matvecs=info.matvecs, err=info.err,
            history=hist)

    def solve_fp64(self, occ, alpha, listmv, d0, kinc, einc, ksc=None, solver=0, tau=0.0,
                   max_step=100, err_max=1e-3, rhs=None, x0=None, want_p=False, trace=True):
        """DDA_FFT in FP64 on the GPU (ddagpu_solve_fp64); returns dict(esc complex128
        (ndir, 3), cabs, cext, steps, step_min, matvecs, err, err_min, trace, p)."""
        o = np.ascontiguousarray(occ, np.int8)
        a = np.ascontiguousarray(np.asarray(alpha, np.complex128)).view(np.float64)
        mv = np.ascontiguousarray(listmv, np.int32)
        ks = np.zeros((0, 3)) if ksc is None else np.ascontiguousarray(np.asarray(ksc, np.float64).reshape(-1, 3))
        nd = ks.shape[0]
        esc = np.zeros((max(nd, 1), 3), np.complex128)
        k = np.ascontiguousarray(kinc, np.float64)
        e = np.ascontiguousarray(np.asarray(einc, np.complex128)).view(np.float64)
        b = None if rhs is None else np.ascontiguousarray(np.asarray(rhs, np.complex128))
        x = None if x0 is None else np.ascontiguousarray(np.asarray(x0, np.complex128))
        p = np.zeros(tuple(self.grid) + (3,), np.complex128) if want_p else None
        tr = np.zeros(max_step + 1) if trace else None
        ca, ce = C.c_double(), C.c_double()
        info = SolveInfo()
        _check(lib().ddagpu_solve_fp64(self._h, solver, tau, _ptr(a), _ptr(mv), len(mv) - 1, _ptr(o),
                                       d0, _ptr(k), _ptr(e), _ptr(b) if b is not None else None,
                                       _ptr(x) if x is not None else None, max_step, err_max, nd,
                                       _ptr(ks), _ptr(esc), C.byref(ca), C.byref(ce),
                                       _ptr(p) if p is not None else None, C.byref(info),
                                       _ptr(tr) if trace else None))
        out = dict(esc=esc[:nd], cabs=ca.value, cext=ce.value, steps=info.steps,
                   step_min=info.step_min if info.rolled_back else -1, matvecs=info.matvecs,
                   err=info.err, err_min=info.err_min, rolled_back=info.rolled_back, p=p)
        if trace:
            out["trace"] = tr[: info.steps + 1]
        return out

    def release_fp64(self):
        _check(lib().ddagpu_release_fp64(self._h))

    def farfield(self, occ, listmv, d0, p, ksc) -> np.ndarray:
        o = np.ascontiguousarray(occ, np.int8)
        mv = np.ascontiguousarray(listmv, np.int32)
        x = _cvec(p)
        ks = _f32(np.asarray(ksc).reshape(-1, 3))
        out = np.zeros((ks.shape[0], 3), np.complex64)
        _check(lib().ddagpu_farfield(self._h, _ptr(mv), len(mv) - 1, _ptr(o), d0, _ptr(x),
                                     ks.shape[0], _ptr(ks), _ptr(out.view(np.float32))))
        return out

    def cabscext(self, occ, alpha, d0, kinc, einc, p):
        o = np.ascontiguousarray(occ, np.int8)
        a = _cvec(np.asarray(alpha, np.complex64).reshape(-1, 1)).ravel()
        x = _cvec(p)
        k = _f32(kinc)      # keep every temporary alive across the call
        e = _cvec(einc)
        ca, ce = C.c_float(), C.c_float()
        _check(lib().ddagpu_cabscext(self._h, d0, _ptr(k), _ptr(e), _ptr(a), len(alpha) - 1,
                                     _ptr(o), _ptr(x), C.byref(ca), C.byref(ce)))
        return ca.value, ce.value

    def mueller(self, kinc, einc0, einc1, ksc, normals, esc0, esc1) -> np.ndarray:
        ks = _f32(ksc)
        npl, nang = ks.shape[:2]
        out = np.zeros((nang, 4, 4), np.float32)
        k, e0, e1, nv = _f32(kinc), _cvec(einc0), _cvec(einc1), _f32(normals)
        s0, s1 = _cvec(esc0), _cvec(esc1)
        _check(lib().ddagpu_mueller(self._h, _ptr(k), _ptr(e0), _ptr(e1), npl, nang, _ptr(ks),
                                    _ptr(nv), _ptr(s0), _ptr(s1), _ptr(out)))
        return out

    def orientation_solves(self, cfg: BatchConfig, rot: np.ndarray):
        """Both polarisations of every orientation rot[k] (3x3), batched on the GPU."""
        rot = np.ascontiguousarray(rot, np.float64).reshape(-1, 3, 3)
        n = rot.shape[0]
        na = num_angles(cfg.theta_min, cfg.theta_max, cfg.theta_step)
        occ = None if cfg.occ is None else np.ascontiguousarray(cfg.occ, np.int8)
        m = np.ascontiguousarray(np.asarray(cfg.materials, np.float32).ravel())
        c = _BatchCfg(cfg.solver, cfg.tau, cfg.max_step, cfg.err_max, cfg.polarizability,
                      len(cfg.materials), _ptr(m), None if occ is None else _ptr(occ),
                      cfg.nplanes, cfg.theta_min, cfg.theta_max, cfg.theta_step)
        cabs = np.zeros(n)
        cext = np.zeros(n)
        mm = np.zeros((n, na, 4, 4))
        info = BatchInfo()
        _check(lib().ddagpu_orientation_solves(self._h, C.byref(c), n, _ptr(rot), _ptr(cabs),
                                               _ptr(cext), _ptr(mm), C.byref(info)))
        return dict(cabs=cabs, cext=cext, mueller=mm, n_rhs=info.n_rhs, max_steps=info.max_steps,
                    rolled_back=info.rolled_back, max_err=info.max_err)

    def _cfg(self, cfg: BatchConfig, m):
        return _BatchCfg(cfg.solver, cfg.tau, cfg.max_step, cfg.err_max, cfg.polarizability,
                         len(cfg.materials), _ptr(m), None, cfg.nplanes, cfg.theta_min,
                         cfg.theta_max, cfg.theta_step)

    def realization_solves(self, cfg: BatchConfig, occ: np.ndarray, rot=None):
        """Both polarisations of every realisation occ[k] (its own occupancy), batched on
        the GPU; rot[k] (3x3) per realisation or None for the fixed orientation."""
        occ = np.ascontiguousarray(occ, np.int8).reshape((-1,) + self.grid)
        n = occ.shape[0]
        r = None if rot is None else np.ascontiguousarray(rot, np.float64).reshape(n, 3, 3)
        na = num_angles(cfg.theta_min, cfg.theta_max, cfg.theta_step)
        m = np.ascontiguousarray(np.asarray(cfg.materials, np.float32).ravel())
        c = self._cfg(cfg, m)
        cabs, cext, mm = np.zeros(n), np.zeros(n), np.zeros((n, na, 4, 4))
        info = BatchInfo()
        _check(lib().ddagpu_realization_solves(self._h, C.byref(c), n, _ptr(occ),
                                               None if r is None else _ptr(r), _ptr(cabs),
                                               _ptr(cext), _ptr(mm), C.byref(info)))
        return dict(cabs=cabs, cext=cext, mueller=mm, n_rhs=info.n_rhs, max_steps=info.max_steps,
                    rolled_back=info.rolled_back, max_err=info.max_err)

    def agglomerate_solves(self, cfg: BatchConfig, monomers, rot=None):
        """Realisations given as monomer lists (Agglomerate.place), rasterised on the GPU
        into the batch; cfg.materials must hold one material."""
        counts = np.array([len(x) for x in monomers], np.int32)
        n = len(counts)
        flat = (np.ascontiguousarray(np.concatenate([np.asarray(x, np.float32).reshape(-1, 13)
                                                     for x in monomers]), np.float32)
                if counts.sum() else np.zeros((1, 13), np.float32))
        r = None if rot is None else np.ascontiguousarray(rot, np.float64).reshape(n, 3, 3)
        na = num_angles(cfg.theta_min, cfg.theta_max, cfg.theta_step)
        m = np.ascontiguousarray(np.asarray(cfg.materials, np.float32).ravel())
        c = self._cfg(cfg, m)
        cabs, cext, mm = np.zeros(n), np.zeros(n), np.zeros((n, na, 4, 4))
        ndip = np.zeros(n, np.int32)
        info = BatchInfo()
        _check(lib().ddagpu_agglomerate_solves(self._h, C.byref(c), n, _ptr(flat), _ptr(counts),
                                               None if r is None else _ptr(r), _ptr(cabs),
                                               _ptr(cext), _ptr(mm), _ptr(ndip), C.byref(info)))
        return dict(cabs=cabs, cext=cext, mueller=mm, ndip=ndip, n_rhs=info.n_rhs,
                    max_steps=info.max_steps, rolled_back=info.rolled_back, max_err=info.max_err)

    # ------------------------------------------------------------ device-resident
    def convolution_dev(self, p_dev, out_dev, nrhs: int = 1, conj: bool = False) -> None:
        """G * p for torch CUDA tensors (nrhs, 3, ni, nj, nl) complex64, on this
        context's stream."""
        _check(lib().ddagpu_convolution_dev(self._h, C.c_void_p(p_dev.data_ptr()),
                                            C.c_void_p(out_dev.data_ptr()), nrhs, int(conj)))

    def set_tiling(self, tile_x=0, rows_g=0):
        _check(lib().ddagpu_set_tiling(self._h, tile_x, rows_g))

    def set_fast_variant(self, x_variant: int = 0, yz_variant: int = 0):
        """Launch variants of the compile-time-sized passes: x 0..11 (tiles, bulk copies,
        second line factorisation, TMA tensor tiles), y/z 0..2 (block sizes)."""
        _check(lib().ddagpu_set_fast_variant(self._h, x_variant, yz_variant))

    def set_farfield_mode(self, mode: int = 0):
        """Far-field form: 0 by kz groups where that halves the work (default), 1 one sum
        per direction, 2 by kz groups whenever possible."""
        _check(lib().ddagpu_set_farfield_mode(self._h, mode))

    @property
    def fast_variant(self):
        x, yz = _i(), _i()
        _check(lib().ddagpu_get_fast_variant(self._h, C.byref(x), C.byref(yz)))
        return x.value, yz.value

    def selftest_wait_timeout(self, on: bool):
        """Diagnostic: make the bulk-copy x pass's bounded wait run out (see the header)."""
        _check(lib().ddagpu_selftest_wait_timeout(self._h, int(on)))

    def set_solver_graph(self, on: bool):
        """Iterations 2..Max_Step of each solve as one CUDA graph launch (default on)."""
        _check(lib().ddagpu_set_solver_graph(self._h, int(on)))

    @property
    def solver_graph_runs(self) -> int:
        return int(lib().ddagpu_solver_graph_runs(self._h))

    def set_kernels(self, fast: bool):
        _check(lib().ddagpu_set_kernels(self._h, int(fast)))

    @property
    def fast_kernels(self) -> bool:
        return lib().ddagpu_get_kernels(self._h) == 1

    def tiling(self):
        a, b = C.c_int(), C.c_int()
        _check(lib().ddagpu_get_tiling(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def autotune(self, nrhs: int = 4):
        _check(lib().ddagpu_autotune(self._h, nrhs))
        return self.tiling()


class Group:
    """Contexts of different lattice sizes whose batched agglomerate solves run as one
    graph launch per call (ddagpu_group_*)."""

    def __init__(self, contexts):
        self.contexts = list(contexts)
        arr = (C.c_void_p * len(self.contexts))(*[c.handle for c in self.contexts])
        h = C.c_void_p()
        _check(lib().ddagpu_group_create(C.byref(h), arr, len(self.contexts)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().ddagpu_group_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def graph_runs(self) -> int:
        return int(lib().ddagpu_group_graph_runs(self._h))

    def agglomerate_solves(self, cfg: BatchConfig, monomers_per_member, rot_per_member=None):
        """monomers_per_member[k]: the monomer lists of member k's realisations (at most its
        max_rhs / 2); returns one result dict per member, as Context.agglomerate_solves."""
        K = len(self.contexts)
        assert len(monomers_per_member) == K
        na = num_angles(cfg.theta_min, cfg.theta_max, cfg.theta_step)
        m = np.ascontiguousarray(np.asarray(cfg.materials, np.float32).ravel())
        c = self.contexts[0]._cfg(cfg, m)
        keep, outs = [], []
        n_real = np.zeros(K, np.int32)
        P = C.c_void_p * K
        mon_p, cnt_p, rot_p, ca_p, ce_p, mm_p, nd_p = P(), P(), P(), P(), P(), P(), P()
        for k, mons in enumerate(monomers_per_member):
            counts = np.array([len(x) for x in mons], np.int32)
            n = len(counts)
            n_real[k] = n
            flat = (np.ascontiguousarray(np.concatenate([np.asarray(x, np.float32).reshape(-1, 13)
                                                         for x in mons]), np.float32)
                    if counts.sum() else np.zeros((1, 13), np.float32))
            out = dict(cabs=np.zeros(max(n, 1)), cext=np.zeros(max(n, 1)),
                       mueller=np.zeros((max(n, 1), na, 4, 4)), ndip=np.zeros(max(n, 1), np.int32))
            r = None
            if rot_per_member is not None and rot_per_member[k] is not None:
                r = np.ascontiguousarray(rot_per_member[k], np.float64).reshape(n, 3, 3)
            keep += [counts, flat, r]
            mon_p[k], cnt_p[k] = flat.ctypes.data, counts.ctypes.data
            rot_p[k] = r.ctypes.data if r is not None else 0
            ca_p[k], ce_p[k] = out["cabs"].ctypes.data, out["cext"].ctypes.data
            mm_p[k], nd_p[k] = out["mueller"].ctypes.data, out["ndip"].ctypes.data
            outs.append(out)
        info = (BatchInfo * K)()
        rots = rot_p if rot_per_member is not None else None
        _check(lib().ddagpu_group_agglomerate_solves(self._h, C.byref(c), _ptr(n_real), mon_p, cnt_p, rots,
                                                     ca_p, ce_p, mm_p, nd_p, info))
        res = []
        for k, out in enumerate(outs):
            n = int(n_real[k])
            res.append(dict(cabs=out["cabs"][:n], cext=out["cext"][:n], mueller=out["mueller"][:n],
                            ndip=out["ndip"][:n], n_rhs=info[k].n_rhs, max_steps=info[k].max_steps,
                            rolled_back=info[k].rolled_back, max_err=info[k].max_err))
        return res
