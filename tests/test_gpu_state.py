"""The sample loop over the batched GPU solves with the reference's state file: configuration
1 end to end against the reference executable's .dat, and the resume rules."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def read_dat(text):
    lines = text.strip().split("\n")
    head = lines[0].replace("\t", " ").split()
    ca, ce = float(head[0].split("=")[1]), float(head[1].split("=")[1])
    rows = np.array([[float(v) for v in ln.split()] for ln in lines[1:]])
    return ca, ce, rows


def test_config1_sample_loop_dat(golden, oracle, tmp_path):
    import dda_fft_b200 as D
    occ, _ = oracle.gen_ellipsoid(32, 32, 32)
    cfg = D.BatchConfig(occ=occ, materials=[(1.5, 0.01)])
    with D.Context(32, 2 * 2.0 / 32, max_rhs=2) as ctx:
        st = D.sample_loop(ctx, cfg, 1, tmp_path / "c1.dst", tmp_path / "c1.dat")
    assert st.counter == 1
    ca, ce, rows = read_dat((tmp_path / "c1.dat").read_text())
    ra, re_, rrows = read_dat(bytes(golden["c1_dat"]).decode())
    assert abs(ca - ra) < 1e-4 * ra and abs(ce - re_) < 3e-4 * re_
    np.testing.assert_array_equal(rows[:, 0], rrows[:, 0])           # theta column
    sig = np.abs(rrows[:, 1:]) > 1e-3 * np.abs(rrows[:, 1:]).max()
    assert (np.abs(rows[:, 1:] - rrows[:, 1:])[sig] / np.abs(rrows[:, 1:])[sig]).max() < 1e-3
    assert (tmp_path / "c1.dst").stat().st_size == len(bytes(golden["c1_dst"]))


def test_resume_repeats_the_stream(oracle, tmp_path):
    """3 Monte-Carlo samples in one run vs 2 + a resumed run to 3: the resumed sample is the
    worker's first draw again (main.cpp:689-690, 803-810)."""
    import dda_fft_b200 as D
    n, x = 16, 2.0
    occ, _ = oracle.gen_ellipsoid(n, n, n, 0.7, 0.5)
    cfg = D.BatchConfig(occ=occ, materials=[(1.55, 0.005)])
    with D.Context(n, 2 * x / n, max_rhs=4) as ctx:
        rot = D.mc_rotations(7, 2)
        r = ctx.orientation_solves(cfg, rot)
        st2 = D.sample_loop(ctx, cfg, 2, tmp_path / "s.dst", orientation="mc", seed=7)
        st3 = D.sample_loop(ctx, cfg, 3, tmp_path / "s.dst", tmp_path / "s.dat",
                            orientation="mc", seed=7)
        one = D.sample_loop(ctx, cfg, 1, tmp_path / "t.dst", orientation="mc", seed=7)
    assert st2.counter == 2 and st3.counter == 3 and one.counter == 1
    want = np.float32(np.float32(r["cabs"][0]) + np.float32(r["cabs"][1]))
    assert abs(st2.cabs - want) <= 1e-5 * want
    assert abs(st3.cabs - (st2.cabs + one.cabs)) <= 1e-5 * st3.cabs
    np.testing.assert_allclose(st3.mueller, st2.mueller + one.mueller, rtol=1e-5,
                               atol=1e-6 * np.abs(st3.mueller).max())
    ca, _, _ = read_dat((tmp_path / "s.dat").read_text())
    assert abs(ca - st3.cabs / 3) <= 1e-6 * ca + 1e-8
    # nothing left to do: the state is unchanged
    with D.Context(n, 2 * x / n, max_rhs=4) as ctx:
        again = D.sample_loop(ctx, cfg, 3, tmp_path / "s.dst", orientation="mc", seed=7)
    assert again.counter == 3 and again.cabs == st3.cabs
