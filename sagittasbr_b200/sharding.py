"""Multi-GPU sharding of a sweep: one process per GPU, no collective on the data path.

Replaces the reference's MPI angle sweep (src/app/sweep.cu:172-179 block partition,
:465-547 MPI_Gather/Gatherv of results, sort by global index, CSV rows).  Every
(angle, frequency) sample is independent, so each rank traces its own contiguous
shard of angles on its own GPU with its own copy of the scene, and the small
results (16 B of field per sample) are gathered once at the end through
torch.distributed (NCCL between GPUs, gloo on CPU-only hosts).

Partitioning can follow the reference exactly (equal angle counts, remainder to
the low ranks) or balance an estimated cost per angle (rays inside the projected
bounding box), which matters when some aspects light up far more of the aperture
than others.
"""
from __future__ import annotations

import math
from typing import Sequence

import numpy as np


def block_partition(n: int, world: int, rank: int) -> tuple[int, int]:
    """(start, count) of the reference's partition: n // world each, the first
    n % world ranks one more (src/app/sweep.cu:172-179)."""
    per, rem = divmod(n, world)
    start = rank * per + min(rank, rem)
    return start, per + (1 if rank < rem else 0)


def cost_partition(costs: Sequence[float], world: int) -> list[tuple[int, int]]:
    """Contiguous (start, count) shards whose summed costs are as even as a prefix
    split allows: shard r ends where the running cost first reaches (r+1)/world of
    the total."""
    c = np.maximum(np.asarray(costs, dtype=np.float64), 0.0)
    n = c.size
    if n == 0:
        return [(0, 0)] * world
    cum = np.cumsum(c)
    total = cum[-1]
    bounds = [0]
    for r in range(1, world):
        if total <= 0:
            b = (n * r) // world
        else:
            b = int(np.searchsorted(cum, total * r / world, side="left")) + 1
        bounds.append(min(max(b, bounds[-1]), n))
    bounds.append(n)
    return [(bounds[r], bounds[r + 1] - bounds[r]) for r in range(world)]


def aperture_cost(aabb_lo, aabb_hi, theta_deg, phi_deg, nx: int, ny: int, grid_size: float) -> np.ndarray:
    """Estimated rays launched per angle: pixels inside the projection of the
    bounding box on the launcher plane (the same clipping the plan applies)."""
    lo = np.asarray(aabb_lo, dtype=np.float64)
    hi = np.asarray(aabb_hi, dtype=np.float64)
    corners = np.array([[hi[0] if c & 1 else lo[0], hi[1] if c & 2 else lo[1], hi[2] if c & 4 else lo[2]]
                        for c in range(8)])
    th = np.radians(np.asarray(theta_deg, dtype=np.float64))
    ph = np.radians(np.asarray(phi_deg, dtype=np.float64))
    d = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], axis=1)
    up = np.where(np.abs(d[:, 1:2]) > 0.99, [[1.0, 0, 0]], [[0, 1.0, 0]])
    u = np.cross(up, d)
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    v = np.cross(d, u)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    s = corners @ u.T / grid_size  # [8, n]
    t = corners @ v.T / grid_size
    ws = np.clip(s.max(0) - s.min(0), 0, 1) * nx + 2
    hs = np.clip(t.max(0) - t.min(0), 0, 1) * ny + 2
    return np.minimum(ws, nx) * np.minimum(hs, ny)


def gather_samples(local_index: np.ndarray, local_values: np.ndarray, n_total: int, group=None):
    """Gathers (global index, values) pairs from every rank to rank 0 and returns the
    values ordered by global index there (None on other ranks)."""
    import torch.distributed as dist
    payload = (np.asarray(local_index, dtype=np.int64), np.asarray(local_values))
    world = dist.get_world_size(group)
    out = [None] * world if dist.get_rank(group) == 0 else None
    dist.gather_object(payload, out, dst=0, group=group)
    if out is None:
        return None
    idx = np.concatenate([o[0] for o in out])
    vals = np.concatenate([o[1] for o in out])
    if idx.size != n_total or np.unique(idx).size != n_total:
        raise RuntimeError("gathered samples do not cover the sweep exactly once")
    order = np.argsort(idx, kind="stable")
    return vals[order]


def shard_of(scene, job, rank: int, world: int, balance: str = "cost") -> list[tuple[int, int]]:
    """(start, count) of every rank's contiguous shard of `job`'s angles: the
    reference's block rule, or balanced by the estimated rays of each angle."""
    th = np.asarray(job.theta_deg, dtype=np.float64)
    ph = np.asarray(job.phi_deg, dtype=np.float64)
    if balance == "cost":
        info = scene.info()
        costs = aperture_cost(info["aabb_lo"], info["aabb_hi"], th, ph, job.nx, job.ny, job.grid_size)
        return cost_partition(costs, world)
    return [block_partition(th.size, world, r) for r in range(world)]


class _DeviceArray:
    """__cuda_array_interface__ view of a device pointer, so torch can wrap a plan's
    result buffer without a copy."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 2,
                                         "strides": None}


class ShardedPlan:
    """One sweep split over the ranks of a process group: this rank's contiguous
    shard of the job's angles as a plan resident on its GPU, and a gather of every
    rank's fields to rank 0 in global angle order straight from device memory
    (all_gather of the padded FP64 field buffers: NCCL over NVLink between GPUs,
    staged through host memory with gloo).  Replaces the reference's MPI partition
    and MPI_Gatherv of results (src/app/sweep.cu:172-179, :465-526)."""

    def __init__(self, scene, job, rank: int, world: int, balance: str = "cost", group=None, **plan_kw):
        import sagittasbr_b200 as sbr
        self.rank, self.world, self.group = rank, world, group
        self.parts = shard_of(scene, job, rank, world, balance)
        self.start, self.count = self.parts[rank]
        self.n_freqs = job.n_freqs
        self.n_angles = int(np.asarray(job.theta_deg).size)
        self.max_count = max(c for _, c in self.parts)
        self.plan = None
        if self.count:
            sl = slice(self.start, self.start + self.count)
            sub = sbr.JobSpec(np.asarray(job.theta_deg, dtype=np.float64)[sl],
                              np.asarray(job.phi_deg, dtype=np.float64)[sl], job.freqs_hz, job.nx, job.ny,
                              job.grid_size, job.max_bounces, job.reflection_const)
            self.plan = sbr.Plan(scene, [sub], **plan_kw)

    def execute(self):
        if self.plan is not None:
            self.plan.execute()

    def gather(self, torch):
        """Every rank's field, on rank 0 as complex128 [n_angles, n_freqs] in angle
        order (None elsewhere).  Collective: every rank calls it."""
        import torch.distributed as dist
        width = self.max_count * self.n_freqs * 2
        dev = torch.device("cuda", torch.cuda.current_device())
        buf = torch.zeros(width, dtype=torch.float64, device=dev)
        if self.plan is not None:
            # the plan may run on a stream of its own: let it finish before the copy
            torch.cuda.synchronize()
            ptr, _ = self.plan.device_results()
            n = self.count * self.n_freqs * 2
            buf[:n].copy_(torch.as_tensor(_DeviceArray(ptr, n), device=dev))
        if dist.get_backend(self.group) == "gloo":
            buf = buf.cpu()
        parts = [torch.empty_like(buf) for _ in range(self.world)]
        dist.all_gather(parts, buf, group=self.group)
        if self.rank != 0:
            return None
        host = [p.cpu().numpy() for p in parts]
        vals = np.concatenate([host[r][:c * self.n_freqs * 2] for r, (_, c) in enumerate(self.parts)])
        if vals.size != self.n_angles * self.n_freqs * 2:
            raise RuntimeError("gathered fields do not cover the sweep exactly once")
        return (vals[0::2] + 1j * vals[1::2]).reshape(self.n_angles, self.n_freqs)

    def close(self):
        if self.plan is not None:
            self.plan.close()
            self.plan = None


def sharded_sweep(scene, job, rank: int, world: int, balance: str = "cost", mode=None, precision=None):
    """Runs this rank's shard of `job`'s angles on its GPU and gathers every
    sample's complex field to rank 0 (returned there in angle order, else None)."""
    import sagittasbr_b200 as sbr
    th = np.asarray(job.theta_deg, dtype=np.float64)
    ph = np.asarray(job.phi_deg, dtype=np.float64)
    n = th.size
    start, count = shard_of(scene, job, rank, world, balance)[rank]
    sl = slice(start, start + count)
    nf = job.n_freqs
    if count:
        sub = sbr.JobSpec(th[sl], ph[sl], job.freqs_hz, job.nx, job.ny, job.grid_size, job.max_bounces,
                          job.reflection_const)
        res = sbr.run(scene, sub, mode=sbr.MODE_BATCHED if mode is None else mode,
                      precision=sbr.PREC_MIXED if precision is None else precision)
        vals = res.field.reshape(count, nf)
    else:
        vals = np.zeros((0, nf), dtype=np.complex128)
    merged = gather_samples(np.arange(start, start + count), vals, n)
    return merged
