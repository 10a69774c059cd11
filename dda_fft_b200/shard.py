"""Samples sharded over ranks (one process per GPU).

Orientations and realisations are independent units (the reference's worker pool,
main.cpp:777-995), so the only exchange is the sum of the per-sample results at the end:
one all-reduce of (Cabs, Cext, Mueller[angles][16]) and the sample count.  Every rank takes
a contiguous range of sample indices; the rotations of all samples are drawn on the host
first from one stream (worker 0's, main.cpp:803-804, 875-898), so the union over ranks is
the single-worker run whatever the rank count.  Sums are kept in FP64 within a rank and
across ranks; the state file (float, written by rank 0) receives them at the end.
"""
from __future__ import annotations

from typing import Callable

import numpy as np


def shard_range(total: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous [start, stop) of `total` samples for `rank` of `world`: the first
    total % world ranks take one sample more."""
    if world < 1 or not 0 <= rank < world or total < 0:
        raise ValueError("bad shard arguments")
    base, extra = divmod(total, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def local_sums(solve: Callable[[np.ndarray], dict], rot: np.ndarray, batch: int) -> dict:
    """Solve this rank's rotations in batches; FP64 sums over its samples."""
    n_angles = None
    out = {"count": 0, "cabs": 0.0, "cext": 0.0, "mueller": None}
    for s0 in range(0, len(rot), batch):
        r = solve(rot[s0:s0 + batch])
        m = np.asarray(r["mueller"], np.float64).reshape(len(r["cabs"]), -1, 4, 4)
        n_angles = m.shape[1]
        out["count"] += len(r["cabs"])
        out["cabs"] += float(np.sum(r["cabs"]))
        out["cext"] += float(np.sum(r["cext"]))
        out["mueller"] = m.sum(0) if out["mueller"] is None else out["mueller"] + m.sum(0)
    if out["mueller"] is None:
        out["mueller"] = np.zeros((0, 4, 4)) if n_angles is None else np.zeros((n_angles, 4, 4))
    return out


def reduce_sums(sums: dict, n_angles: int, group=None, device=None) -> dict:
    """All-reduce of one rank's sums (torch.distributed, any backend): the job's sums on
    every rank."""
    import torch
    import torch.distributed as dist
    m = sums["mueller"] if len(sums["mueller"]) else np.zeros((n_angles, 4, 4))
    flat = np.concatenate([[sums["count"], sums["cabs"], sums["cext"]], np.ravel(m)])
    t = torch.tensor(flat, dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    v = t.cpu().numpy()
    return {"count": int(round(v[0])), "cabs": float(v[1]), "cext": float(v[2]),
            "mueller": v[3:].reshape(n_angles, 4, 4)}


def sharded_sample_sums(solve: Callable[[np.ndarray], dict], rot_all: np.ndarray, n_angles: int,
                        rank: int, world: int, batch: int, group=None, device=None) -> dict:
    """This rank's contiguous share of rot_all solved through `solve` (a batched call such as
    Context.orientation_solves bound to a configuration), then the all-reduce."""
    a, b = shard_range(len(rot_all), world, rank)
    return reduce_sums(local_sums(solve, rot_all[a:b], batch), n_angles, group, device)


def write_state(sums: dict, state_path: str, dat_path: str | None, theta_min: float,
                theta_step: float) -> None:
    """Rank 0 stores the reduced sums as the reference's state (and .dat)."""
    from .api import StateFile
    n_angles = sums["mueller"].shape[0]
    st = StateFile(state_path, n_angles, restart=True)
    st.counter = sums["count"]
    st.cabs = float(np.float32(sums["cabs"]))
    st.cext = float(np.float32(sums["cext"]))
    st.mueller[...] = sums["mueller"].astype(np.float32)
    st.save()
    if dat_path is not None and st.counter > 0:
        st.write_dat(dat_path, theta_min, theta_step)
