"""PALMAD and PD3 sharded over the GPUs of a job, one process (or thread) each.

The reference splits the series into one fragment per GPU with an
(maxL - 1) halo (src/data_preparation.cuh:30-75), runs phase 1 per fragment,
exchanges the candidates all-to-all (src/MPI_transfers.hpp:29-84), refines
every candidate against every fragment and takes the minimum distance over
the GPUs (src/sets_processing.hpp:152-164).  Here every rank holds the whole
series (8 MB at n = 2^21) and an attempt (length m, threshold r) is:

1. phase 1 on the rank's rows; the alive flags of all windows are combined
   with an element-wise minimum (AND) over the ranks;
2. the refine of the combined candidates against the rank's columns (a range
   of the 2048-window tile grid); per candidate the correlation maximum (an
   order-preserving uint32 image) and the pruned flag are combined with a
   maximum over the ranks;
3. classification, FP64 recheck and top-k on every rank (identical results).

The per-rank compute is a *backend* (``GpuBackend`` runs libpaddi's
``paddi_shard_*`` entry points); the exchanges go through a *communicator*
(``TorchComm``: torch.distributed, NCCL between GPUs or gloo on CPU;
``ThreadComm``: ranks as threads of one process).  The r-schedule is the
library's own (``paddi_merlin_first_r`` / ``paddi_merlin_lower``), so the
attempts are those of a single-GPU MERLIN run.

No TMA or bulk load reads another GPU's memory: every exchange is a
collective on buffers the ranks own.
"""
from __future__ import annotations

import ctypes as C
import threading

import numpy as np

from . import (Discord, PaddiError, PADDI_OK, _Discord, _Log, lib)

TILE = 2048  # column shards start on the refine's tile grid


def shard_ranges(N: int, world: int, grid: int = TILE):
    """(rows, cols): per rank a [lo, hi) range of windows for phase 1 and for
    the refine; column edges on the tile grid (the last one is N)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    cuts = [min(N, (N * k // world) // grid * grid) for k in range(world + 1)]
    cuts[-1] = N
    cols = [(cuts[k], cuts[k + 1]) for k in range(world)]
    rows = [(N * k // world, N * (k + 1) // world) for k in range(world)]
    return rows, cols


def merlin_first_r(out, j: int, minL: int):
    """The reference schedule's first r of length minL + j and its decrement S."""
    n = max(j, 1)
    arr = (_Discord * n)()
    for i in range(j):
        arr[i].ind, arr[i].dist = int(out[i][0]), float(out[i][1])
    S = C.c_float(0.0)
    r = lib().paddi_merlin_first_r(arr, j, minL, C.byref(S))
    return float(r), float(S.value)


def merlin_lower(r: float, j: int, S: float) -> float:
    return float(lib().paddi_merlin_lower(float(r), j, float(S)))


# ---------------------------------------------------------------- communicators
class TorchComm:
    """Exchanges over a torch.distributed process group (NCCL or gloo).

    device: where the collective tensors live ('cuda:<i>' for NCCL, 'cpu' for
    gloo)."""

    def __init__(self, group=None, device="cpu"):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.device = device
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    def all_min_u8(self, t):
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MIN, group=self.group)
        return t

    def all_gather(self, t):
        import torch
        out = [torch.empty_like(t) for _ in range(self.world)]
        self.dist.all_gather(out, t, group=self.group)
        return out


class ThreadComm:
    """``world`` ranks as threads of one process (one GPU or CPU): each
    exchange is a barrier around a shared slot list."""

    class _Shared:
        def __init__(self, world):
            self.world = world
            self.barrier = threading.Barrier(world)
            self.slots = [None] * world

    def __init__(self, shared: "ThreadComm._Shared", rank: int):
        self.s = shared
        self.rank = rank
        self.world = shared.world

    @classmethod
    def group(cls, world: int):
        sh = cls._Shared(world)
        return [cls(sh, r) for r in range(world)]

    def _exchange(self, t):
        self.s.slots[self.rank] = t.clone()
        self.s.barrier.wait()
        got = list(self.s.slots)
        self.s.barrier.wait()
        return got

    def all_min_u8(self, t):
        got = self._exchange(t)
        out = got[0]
        for g in got[1:]:
            out = out.minimum(g)
        t.copy_(out)
        return t

    def all_gather(self, t):
        return self._exchange(t)


def merge_candidates(comm, ind, rho, pruned):
    """Per window, the maximum of rho and of pruned over the ranks.  Every rank
    holds the same candidate set in an order of its own: each rank's arrays
    are sorted by window, then combined element-wise.  ind int32, rho int64
    (the uint32 order image), pruned uint8; torch tensors."""
    import torch
    order = torch.argsort(ind.to(torch.int64))
    ind, rho, pruned = ind[order], rho[order], pruned[order]
    if comm is None or comm.world == 1:
        return ind, rho, pruned
    n = torch.tensor([ind.numel()], dtype=torch.int64, device=ind.device)
    counts = comm.all_gather(n)
    if any(int(c.item()) != ind.numel() for c in counts):
        raise RuntimeError("ranks disagree on the candidate set size")
    inds = comm.all_gather(ind.contiguous())
    rhos = comm.all_gather(rho.contiguous())
    prs = comm.all_gather(pruned.contiguous())
    for i2 in inds:
        if not torch.equal(i2, ind):
            raise RuntimeError("ranks disagree on the candidate set")
    rho_m = torch.stack(rhos).amax(dim=0)
    pr_m = torch.stack(prs).amax(dim=0)
    return ind, rho_m, pr_m


# ---------------------------------------------------------------- GPU backend
class GpuBackend:
    """One rank's compute: a libpaddi context and the series on its device."""

    def __init__(self, ctx, series, device: int = 0):
        import torch
        self.torch = torch
        self.ctx = ctx
        self.dev = f"cuda:{device}"
        self.x = torch.as_tensor(np.ascontiguousarray(series, np.float32)).to(self.dev)
        self.n = int(self.x.numel())

    def phase1(self, m, r2, lo, hi):
        torch = self.torch
        N = self.n - m + 1
        alive = torch.empty(N, dtype=torch.uint8, device=self.dev)
        self.ctx._check(lib().paddi_shard_phase1(self.ctx._h, C.c_void_p(self.x.data_ptr()),
                                                 self.n, m, C.c_float(r2), lo, hi,
                                                 C.c_void_p(alive.data_ptr())))
        return alive

    def refine(self, m, r2, alive, lo, hi):
        torch = self.torch
        N = self.n - m + 1
        ind = torch.empty(N, dtype=torch.int32, device=self.dev)
        rho = torch.empty(N, dtype=torch.int32, device=self.dev)  # uint32 bits
        pr = torch.empty(N, dtype=torch.uint8, device=self.dev)
        cnt = C.c_uint32(0)
        self.ctx._check(lib().paddi_shard_refine(
            self.ctx._h, C.c_void_p(self.x.data_ptr()), self.n, m, C.c_float(r2),
            C.c_void_p(alive.data_ptr()), lo, hi, C.c_void_p(ind.data_ptr()),
            C.c_void_p(rho.data_ptr()), C.c_void_p(pr.data_ptr()), N, C.byref(cnt)))
        c = cnt.value
        return ind[:c], rho[:c].to(torch.int64) & 0xFFFFFFFF, pr[:c]

    def select(self, m, r2, ind, rho, pruned, top_k):
        torch = self.torch
        ind = ind.to(self.dev, torch.int32).contiguous()
        r32 = rho.to(self.dev)
        r32 = torch.where(r32 >= 2 ** 31, r32 - 2 ** 32, r32).to(torch.int32).contiguous()
        pruned = pruned.to(self.dev, torch.uint8).contiguous()
        out = (_Discord * 16)()
        n_out = C.c_uint32(0)
        log = _Log()
        self.ctx._check(lib().paddi_shard_select(
            self.ctx._h, C.c_void_p(self.x.data_ptr()), self.n, m, C.c_float(r2),
            C.c_void_p(ind.data_ptr()), C.c_void_p(r32.data_ptr()),
            C.c_void_p(pruned.data_ptr()), int(ind.numel()), top_k, out, C.byref(n_out),
            C.byref(log)))
        return [(out[i].ind, out[i].dist) for i in range(n_out.value)], log.as_dict()


# ---------------------------------------------------------------- drivers
def attempt_sharded(backend, comm, m: int, r2: float, top_k: int = 1):
    """One (m, r2) attempt over the ranks; every rank returns the same result."""
    rank = comm.rank if comm is not None else 0
    world = comm.world if comm is not None else 1
    N = backend.n - m + 1
    rows, cols = shard_ranges(N, world)
    alive = backend.phase1(m, r2, *rows[rank])
    if world > 1:
        comm.all_min_u8(alive)
    if cols[rank][0] < cols[rank][1]:
        ind, rho, pr = backend.refine(m, r2, alive, *cols[rank])
    else:  # more ranks than tiles: this rank's column range is empty
        ind, rho, pr = backend.refine(m, r2, alive, 0, min(N, TILE))
        rho = rho * 0
        pr = pr * 0
    ind, rho, pr = merge_candidates(comm, ind, rho, pr)
    return backend.select(m, r2, ind, rho, pr, top_k)


def palmad_sharded(backend, comm, minL: int, maxL: int, iter_cap: int = 200):
    """Top-1 discord of every length minL..maxL with the reference's MERLIN
    schedule (src/main.cu:136-233), each attempt sharded over the ranks.
    Returns ([Discord], [attempt log dicts])."""
    out, logs = [], []
    for j in range(maxL - minL + 1):
        m = minL + j
        r, S = merlin_first_r(out, j, minL)
        for it in range(iter_cap + 1):
            if it == iter_cap:
                raise PaddiError(4, f"length {m}: no discord after {iter_cap} attempts")
            r32 = np.float32(r)
            r2 = float(r32 * r32)
            sel, log = attempt_sharded(backend, comm, m, r2, 1)
            log["r"] = float(r32)
            logs.append(log)
            if sel:
                out.append(sel[0])
                break
            r = merlin_lower(float(r32), j, S)
    return [Discord(int(i), float(d)) for i, d in out], logs


def pd3_sharded(backend, comm, m: int, top_k: int = 1, iter_cap: int = 200):
    """Fixed-length top-k discords with the halving schedule from 2 sqrt(m)
    (src/main.cu:136-156), each attempt sharded over the ranks."""
    r = np.float32(2.0 * np.sqrt(float(m)))
    logs = []
    for _ in range(iter_cap):
        r2 = float(r * r)
        sel, log = attempt_sharded(backend, comm, m, r2, top_k)
        logs.append(log)
        if len(sel) >= top_k or r2 == 0.0:
            return [Discord(int(i), float(d)) for i, d in sel], logs
        r = np.float32(0.5 * float(r))
    raise PaddiError(4, "no discords after the attempt cap")


__all__ = ["shard_ranges", "TorchComm", "ThreadComm", "GpuBackend", "merge_candidates",
           "attempt_sharded", "palmad_sharded", "pd3_sharded", "merlin_first_r",
           "merlin_lower", "PADDI_OK"]
