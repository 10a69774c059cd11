"""Realisations on lattices of different sizes as ONE graph launch (ddagpu_group_*), against
the same realisations solved by each lattice's context on its own: the same kernels on the
same inputs, so the results are bit-identical."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = (32, 64, 128)
X, MAT, R, RHO = 6.0, (1.55, 0.005), 3.0, 0.25


def realisations(D, n, count, seed):
    c = D.Agglomerate.count((n, n, n), RHO, R, 0.0)
    return [D.Agglomerate(seed, k).place(n, R, 0.0, c) for k in range(count)]


def test_group_matches_members_bit_for_bit():
    import dda_fft_b200 as D
    cfg = D.BatchConfig(occ=None, materials=[MAT], nplanes=2)
    ctxs = [D.Context(n, 2 * X / n, max_rhs=8) for n in SIZES]
    mons = [realisations(D, n, 3, 7 + n) for n in SIZES]
    rots = [D.mc_rotations(11, 3, k) for k in range(len(SIZES))]
    alone = [c.agglomerate_solves(cfg, m, r) for c, m, r in zip(ctxs, mons, rots)]
    with D.Group(ctxs) as grp:
        for call in range(2):           # the second call replays the recorded graph
            runs = grp.graph_runs
            together = grp.agglomerate_solves(cfg, mons, rots)
            assert grp.graph_runs == runs + 1
            for a, t in zip(alone, together):
                for q in ("cabs", "cext", "mueller", "ndip"):
                    assert np.array_equal(a[q], t[q]), q
                assert a["max_steps"] == t["max_steps"]
        # a member left out, another solve shape (fixed orientation): the graph is rebuilt
        part = grp.agglomerate_solves(cfg, [mons[0], [], mons[2]])
        assert len(part[1]["cabs"]) == 0
        for k in (0, 2):
            ref = ctxs[k].agglomerate_solves(cfg, mons[k])
            assert np.array_equal(ref["mueller"], part[k]["mueller"])
    for c in ctxs:
        c.close()


def test_group_rejects_oversized_batches():
    import dda_fft_b200 as D
    cfg = D.BatchConfig(occ=None, materials=[MAT])
    ctxs = [D.Context(32, 2 * X / 32, max_rhs=2), D.Context(64, 2 * X / 64, max_rhs=2)]
    with D.Group(ctxs) as grp:
        with pytest.raises(D.DDAGPUError):
            grp.agglomerate_solves(cfg, [realisations(D, 32, 2, 1), []])
    with pytest.raises(D.DDAGPUError):
        D.Group([ctxs[0], ctxs[0]])
    for c in ctxs:
        c.close()
