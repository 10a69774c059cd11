"""CPU checks of the C-ABI library: it builds for sm_100a, loads, exports every function
include/ddagpu.h declares, and its host-only helpers agree with the oracle.  No kernel is
launched here."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "ddagpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ddagpu_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from dda_fft_b200 import lib
    L = lib()
    syms = declared_symbols()
    assert len(syms) >= 19
    for s in syms:
        assert hasattr(L, s), s
    assert b"sm_100a" in L.ddagpu_version()


def test_library_is_built_for_sm100a_only():
    """The build recipe targets sm_100a and nothing else; the loaded module itself is
    checked at run time by test_kernels_report_sm100, on a GPU."""
    mk = open(os.path.join(ROOT, "dda_fft_b200", "csrc", "Makefile")).read()
    arch = re.findall(r"-gencode\s+arch=(\S+),code=(\S+)", mk)
    assert arch == [("compute_100a", "sm_100a")]


@pytest.mark.gpu
def test_kernels_report_sm100():
    from dda_fft_b200 import lib
    v = C.c_int(0)
    assert lib().ddagpu_binary_version(0, C.byref(v)) == 0, lib().ddagpu_last_error()
    assert v.value == 100


def test_create_fails_loudly_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from dda_fft_b200 import Context, DDAGPUError
    with pytest.raises(DDAGPUError):
        Context(8, 0.5)


def test_bad_arguments_rejected():
    from dda_fft_b200 import lib
    L = lib()
    h = C.c_void_p()
    assert L.ddagpu_create(C.byref(h), 0, 12, 8, 8, 0.5, 1) == -1      # not a power of two
    assert L.ddagpu_create(C.byref(h), 0, 256, 8, 8, 0.5, 1) == -1     # above 128
    assert L.ddagpu_create(C.byref(h), 0, 8, 8, 8, -1.0, 1) == -1      # kd <= 0
    assert L.ddagpu_create(None, 0, 8, 8, 8, 0.5, 1) == -1


def test_mc_rotations_match_reference_sampler(oracle):
    from dda_fft_b200 import mc_rotations
    for seed, worker in ((7, 0), (1, 3), (0, 0)):
        T = mc_rotations(seed, 16, worker)
        To = oracle.mc_rotations(seed, worker, 16)
        assert np.abs(T - To).max() < 1e-12
        for t in T:
            assert np.abs(t @ t.T - np.eye(3)).max() < 1e-12


def test_fixed_rotation_and_angles():
    from dda_fft_b200 import fixed_rotation, num_angles
    assert np.abs(fixed_rotation(0, 0, 0) - np.eye(3)).max() < 1e-15
    T = fixed_rotation(30.0, 45.0, 60.0)
    assert np.abs(T @ T.T - np.eye(3)).max() < 1e-12
    assert num_angles(0, 180, 10) == 19
    assert num_angles(0, 180, 1) == 181
    assert num_angles(0, 180, 2) == 91


def test_new_entry_points_reject_bad_arguments_without_a_device():
    """The FP64 solve, groups, the far-field mode and the architecture query fail loudly on
    bad arguments (and, on a machine without a GPU, report that instead of computing
    anything)."""
    import torch
    from dda_fft_b200 import lib
    L = lib()
    h = C.c_void_p()
    assert L.ddagpu_group_create(C.byref(h), None, 0) == -1
    assert L.ddagpu_group_create(None, None, 1) == -1
    assert L.ddagpu_group_destroy(None) == 0
    assert L.ddagpu_group_graph_runs(None) == -1
    z = C.c_double()
    assert L.ddagpu_solve_fp64(None, 0, 0.0, None, None, 1, None, 0.5, None, None, None, None, 5, 1e-3,
                               0, None, None, C.byref(z), C.byref(z), None, None, None) == -1
    assert L.ddagpu_release_fp64(None) == -1
    assert L.ddagpu_set_farfield_mode(None, 0) == -1
    v = C.c_int(0)
    assert L.ddagpu_binary_version(0, None) == -1
    if not torch.cuda.is_available():
        assert L.ddagpu_binary_version(0, C.byref(v)) == -5      # DDAGPU_ENOTBUILT
