"""Samples sharded over ranks: contiguous ranges, one all-reduce of the sums at the end,
and the state written by rank 0.  Two gloo ranks on the CPU with a deterministic stand-in
for the batched GPU call (the solves themselves are covered by the GPU parity tests)."""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

N_ANGLES = 5


def fake_solve(rot):
    """A deterministic function of each rotation, shaped like Context.orientation_solves."""
    rot = np.asarray(rot)
    n = len(rot)
    cabs = rot[:, 0, 0] + 2 * rot[:, 1, 2]
    cext = 1 + rot[:, 2, 2] ** 2
    mm = np.einsum("nij,a->naij", np.pad(rot, ((0, 0), (0, 1), (0, 1))), np.arange(1, N_ANGLES + 1))
    return {"cabs": cabs, "cext": cext, "mueller": mm.reshape(n, N_ANGLES, 4, 4)}


@pytest.mark.parametrize("total", [0, 1, 5, 16, 17])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shard_range_partitions(total, world):
    from dda_fft_b200.shard import shard_range
    spans = [shard_range(total, world, r) for r in range(world)]
    assert spans[0][0] == 0 and spans[-1][1] == total
    for (a, b), (c, _) in zip(spans, spans[1:]):
        assert b == c
    sizes = [b - a for a, b in spans]
    assert max(sizes) - min(sizes) <= 1


def _rank(rank, world, port, outdir):
    import torch.distributed as dist
    from dda_fft_b200 import mc_rotations
    from dda_fft_b200.shard import sharded_sample_sums, write_state
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    rot = mc_rotations(7, 11)
    s = sharded_sample_sums(fake_solve, rot, N_ANGLES, rank, world, batch=2)
    np.save(os.path.join(outdir, f"r{rank}.npy"),
            np.concatenate([[s["count"], s["cabs"], s["cext"]], s["mueller"].ravel()]))
    if rank == 0:
        write_state(s, os.path.join(outdir, "s.dst"), os.path.join(outdir, "s.dat"), 0.0, 45.0)
    dist.barrier()
    dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_equal_one_worker():
    from dda_fft_b200 import StateFile, mc_rotations
    from dda_fft_b200.shard import local_sums
    with tempfile.TemporaryDirectory() as d:
        mp.spawn(_rank, args=(2, free_port(), d), nprocs=2, join=True)
        r0, r1 = (np.load(os.path.join(d, f"r{k}.npy")) for k in range(2))
        np.testing.assert_array_equal(r0, r1)             # every rank holds the job's sums
        ref = local_sums(fake_solve, mc_rotations(7, 11), batch=3)
        assert r0[0] == 11 == ref["count"]
        assert abs(r0[1] - ref["cabs"]) < 1e-12 and abs(r0[2] - ref["cext"]) < 1e-12
        np.testing.assert_allclose(r0[3:], ref["mueller"].ravel(), rtol=0, atol=1e-12)
        st = StateFile(os.path.join(d, "s.dst"), N_ANGLES)
        assert st.counter == 11 and st.cabs == np.float32(ref["cabs"])
        np.testing.assert_array_equal(st.mueller, ref["mueller"].astype(np.float32))
        assert os.path.getsize(os.path.join(d, "s.dat")) > 0


def test_single_process_without_group():
    """Without an initialised process group the reduction is the identity."""
    from dda_fft_b200 import mc_rotations
    from dda_fft_b200.shard import local_sums, sharded_sample_sums
    rot = mc_rotations(3, 4)
    s = sharded_sample_sums(fake_solve, rot, N_ANGLES, 0, 1, batch=4)
    ref = local_sums(fake_solve, rot, batch=1)
    assert s["count"] == 4 and abs(s["cabs"] - ref["cabs"]) < 1e-12
