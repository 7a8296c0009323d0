"""Multi-GPU plumbing of the trace: one process per GPU, the sun-ray index range split
contiguously over the ranks, the exchanges done through torch.distributed.

st_sim_run on N ranks (st_b200_set_ranks) gives exactly the results of one run on one
GPU: every ray keeps its random stream (key: the run seed; counter: its global sun-ray
index), rank r traces a contiguous slice of each batch's sun-ray range, ray numbers are the
rank's hit ranks offset by an exclusive prefix of the ranks' hit counts, and the run stops at
the same hit.  The library asks the caller for two collectives, which RankExchange
implements over torch.distributed ("gloo" with CPU tensors, "nccl" with CUDA tensors):

  allgather(send[count] -> recv[count * nranks], rank-major): the ranks' hit counts per
      batch (one 64-bit number each), before the batch's hits are numbered and traced;
  allreduce(buf[count], op): at the end of the run, the integer flux bins, per-element
      counters and stage counters summed (op 0) and SunRayCount, the largest ray numbers
      and the flags reduced with max (op 1) -- exact and independent of the rank count.

Records stay with the rank that traced them (its st_locations & co. return its own rays,
numbered globally).  The reference's multi-thread convention it replaces runs independent
contexts with seeds seed + i*123 and concatenates them (app/src/trace.cpp:709-735,
pysoltrace.py:1615-1661); here the ranks together make one run.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

_u64p = C.POINTER(C.c_ulonglong)
ALLGATHER_FN = C.CFUNCTYPE(C.c_int, _u64p, _u64p, C.c_int, C.c_void_p)
ALLREDUCE_FN = C.CFUNCTYPE(C.c_int, _u64p, C.c_ulonglong, C.c_int, C.c_void_p)
OP_SUM, OP_MAX = 0, 1


def _dist():
    try:
        import torch.distributed as dist
    except ImportError:  # pragma: no cover - torch is part of the image
        return None
    return dist if dist.is_available() and dist.is_initialized() else None


class RankExchange:
    """The two collectives st_sim_run needs, over the default torch.distributed group (or
    `group`).  `device` is where the collective's tensors live: "cpu" for gloo, "cuda" for
    NCCL.  Values are 64-bit counts, carried as int64 (every count stays below 2^63)."""

    def __init__(self, device: str = "cpu", group=None):
        import torch
        self.torch = torch
        self.dist = _dist()
        if self.dist is None:
            raise RuntimeError("torch.distributed is not initialised")
        self.device = device
        self.group = group
        self.rank = self.dist.get_rank(group)
        self.world = self.dist.get_world_size(group)
        self.errors = []
        # the C callbacks (kept alive with this object)
        self.c_allgather = ALLGATHER_FN(self._allgather)
        self.c_allreduce = ALLREDUCE_FN(self._allreduce)

    def allgather(self, send: np.ndarray) -> np.ndarray:
        t = self.torch.from_numpy(np.ascontiguousarray(send, dtype=np.int64)).to(self.device)
        out = self.torch.empty(self.world * t.numel(), dtype=self.torch.int64, device=self.device)
        self.dist.all_gather_into_tensor(out, t, group=self.group)
        return out.cpu().numpy()

    def allreduce(self, buf: np.ndarray, op: int) -> np.ndarray:
        t = self.torch.from_numpy(np.ascontiguousarray(buf, dtype=np.int64)).to(self.device)
        red = self.dist.ReduceOp.SUM if op == OP_SUM else self.dist.ReduceOp.MAX
        self.dist.all_reduce(t, op=red, group=self.group)
        return t.cpu().numpy()

    def _allgather(self, send, recv, count, user):
        try:
            s = np.ctypeslib.as_array(send, shape=(count,)).view(np.int64)
            r = np.ctypeslib.as_array(recv, shape=(count * self.world,)).view(np.int64)
            r[:] = self.allgather(s)
            return 1
        except Exception as ex:  # noqa: BLE001 - reported to the library as a failed exchange
            self.errors.append(repr(ex))
            return 0

    def _allreduce(self, buf, count, op, user):
        try:
            b = np.ctypeslib.as_array(buf, shape=(int(count),)).view(np.int64)
            b[:] = self.allreduce(b, int(op))
            return 1
        except Exception as ex:  # noqa: BLE001
            self.errors.append(repr(ex))
            return 0

    def attach(self, api, ctx) -> int:
        """st_b200_set_ranks(ctx, rank, world, allgather, allreduce): the context's runs are
        this rank's share of one run over all ranks."""
        return api.st_b200_set_ranks(ctx, self.rank, self.world, self.c_allgather, self.c_allreduce, None)


def combine(units: float, dev_ms: float, wall_ms: float, device: str = "cpu"):
    """Whole-job timing of a sharded run: units are already the run's (identical on every
    rank); device and wall times are the max over ranks (the job takes as long as its
    slowest rank)."""
    dist = _dist()
    if dist is None or dist.get_world_size() == 1:
        return float(units), float(dev_ms), float(wall_ms)
    import torch
    m = torch.tensor([float(dev_ms), float(wall_ms)], dtype=torch.float64, device=device)
    dist.all_reduce(m, op=dist.ReduceOp.MAX)
    return float(units), m[0].item(), m[1].item()
