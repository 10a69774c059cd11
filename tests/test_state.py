"""State (.dst) and result (.dat) files against the reference executable's own files for
configuration 1 (tests/golden: c1_dst, c1_dat written by the unmodified reference): the
layout, the text format and the resume rules (main.cpp:214-274, 961-981, 1085-1118).
No kernel runs here."""
import struct

import numpy as np
import pytest


def golden_state(golden):
    raw = bytes(golden["c1_dst"])
    counter, cabs, cext = struct.unpack("<iff", raw[:12])
    mm = np.frombuffer(raw[12:], np.float32).reshape(-1, 4, 4)
    return raw, counter, cabs, cext, mm


def test_dat_is_byte_exact(golden, tmp_path):
    """The .dat written from the reference's own .dst equals the reference's .dat."""
    from dda_fft_b200 import StateFile
    raw, counter, cabs, cext, mm = golden_state(golden)
    dst = tmp_path / "c1.dst"
    dst.write_bytes(raw)
    st = StateFile(dst, mm.shape[0])
    assert (st.counter, st.cabs, st.cext) == (counter, cabs, cext)
    np.testing.assert_array_equal(st.mueller, mm)
    st.write_dat(tmp_path / "c1.dat", 0.0, 10.0)
    assert (tmp_path / "c1.dat").read_bytes() == bytes(golden["c1_dat"])


def test_dst_round_trip_is_byte_exact(golden, tmp_path):
    from dda_fft_b200 import StateFile
    raw, *_ , mm = golden_state(golden)
    src = tmp_path / "a.dst"
    src.write_bytes(raw)
    st = StateFile(src, mm.shape[0])
    st.path = str(tmp_path / "b.dst")
    st.save()
    assert (tmp_path / "b.dst").read_bytes() == raw


def test_fresh_restart_and_short_state(tmp_path):
    from dda_fft_b200 import DDAGPUError, StateFile
    p = tmp_path / "s.dst"
    st = StateFile(p, 19)                       # created with a zero state
    assert st.counter == 0 and st.cabs == 0 and not st.mueller.any()
    assert p.stat().st_size == 12 + 19 * 64
    st.counter, st.cabs = 5, 1.25
    st.save()
    assert StateFile(p, 19).counter == 5        # resumed
    assert StateFile(p, 19, restart=True).counter == 0
    with pytest.raises(DDAGPUError):            # fewer angles stored than asked for
        StateFile(p, 40)


def test_accumulate_in_float_in_order(tmp_path):
    """Samples add to float sums one after another, like the reference's accumulation."""
    from dda_fft_b200 import StateFile
    rng = np.random.default_rng(1)
    n, na = 7, 3
    res = {"cabs": rng.random(n) * 3, "cext": rng.random(n) * 1e3,
           "mueller": rng.standard_normal((n, na, 4, 4))}
    st = StateFile(tmp_path / "x.dst", na)
    st.add({k: v[:3] for k, v in res.items()})
    st.add({k: v[3:] for k, v in res.items()})
    ca, ce, mm = np.float32(0), np.float32(0), np.zeros((na, 4, 4), np.float32)
    for s in range(n):
        ca = np.float32(ca + np.float32(res["cabs"][s]))
        ce = np.float32(ce + np.float32(res["cext"][s]))
        mm = (mm + res["mueller"][s].astype(np.float32)).astype(np.float32)
    assert st.counter == n and st.cabs == ca and st.cext == ce
    np.testing.assert_array_equal(st.mueller, mm)


def test_bad_arguments(tmp_path):
    from dda_fft_b200 import DDAGPUError, lib
    L = lib()
    assert L.ddagpu_write_dat(str(tmp_path / "z.dat").encode(), 0, 0, 0, 0, 0, 1, None) != 0
    with pytest.raises(DDAGPUError):
        from dda_fft_b200.api import _check
        _check(L.ddagpu_state_write(b"/nonexistent-dir/x.dst", 0, 0, 0, 0, None))
