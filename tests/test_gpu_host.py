"""The reference's own executable with its DDA_FFT call sent to libddagpu.

oracle/_ref/dda_fft_gpu.out is the reference's main.cpp with oracle/main_ddagpu.patch
applied (one ddagpu context per worker, ddagpu_dda_fft in place of DDA_FFT at
main.cpp:933-937), compiled against include/ddagpu.h and linked to libddagpu.so by
oracle/Makefile.  Config 1 runs through it with the reference's own command line; its .dat
and .dst must have the executable's layout (same lines, same angle column, same byte size)
and numbers within the float-parity gate of the executable's own .dat (tests/golden c1_dat,
made by the unmodified executable)."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "dda_fft_gpu.out")
C1 = ["--target", "sphere", "--grid", "32", "-x", "2", "-m", "1.5", "0.01", "-P", "cm", "-M", "cg",
      "-e", "1e-3", "-S", "20", "--orientation", "fixed", "--planes", "1", "-a", "0", "-b", "180",
      "-s", "10", "--seed", "1", "--threads", "1", "--restart"]


def parse(txt):
    lines = txt.strip().split("\n")
    head = lines[0].replace("\t", " ").split()
    rows = np.array([[float(v) for v in ln.split()] for ln in lines[1:]])
    return float(head[0].split("=")[1]), float(head[1].split("=")[1]), rows, lines


def test_reference_host_through_libddagpu(golden, tmp_path):
    if not os.path.exists(EXE):
        pytest.skip("oracle/_ref/dda_fft_gpu.out not built (needs the reference tree)")
    out = subprocess.run([EXE] + C1 + ["-o", "c1.dat", "-D", "c1.dst"], cwd=tmp_path,
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    got = (tmp_path / "c1.dat").read_text()
    ref = bytes(golden["c1_dat"]).decode()
    ca, ce, rows, lines = parse(got)
    ca0, ce0, rows0, lines0 = parse(ref)
    assert len(lines) == len(lines0)
    assert lines[0].split("=")[0] == lines0[0].split("=")[0]
    assert np.array_equal(rows[:, 0], rows0[:, 0])                 # the angle column
    assert os.path.getsize(tmp_path / "c1.dst") == len(golden["c1_dst"])
    assert abs(ca - ca0) < 1e-4 * ca0
    assert abs(ce - ce0) < 3e-4 * ce0       # the float reference's own noise on Cext here
    M, M0 = rows[:, 1:], rows0[:, 1:]
    sig = np.abs(M0) > 1e-3 * np.abs(M0).max()
    assert (np.abs(M - M0)[sig] / np.abs(M0)[sig]).max() < 1e-3
