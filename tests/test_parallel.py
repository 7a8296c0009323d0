"""Host side of runs over several ranks (st_b200_set_ranks), as two gloo ranks on the CPU.

`soltrace_b200.parallel.RankExchange` supplies the two collectives st_sim_run calls on every
rank of a sharded run: an all-gather of the ranks' hit counts per sun-ray batch and, at the
end, all-reduces (sum, max) of the run's counters and flux maps.  Here two processes bind it
over gloo and call the C callbacks exactly as the library does (through ctypes function
pointers, on 64-bit buffers), check rank-major gathering and both reductions, set the ranks on
the product library's contexts (and have bad rank arguments refused), and check that without
a GPU both ranks' st_sim_run fail at once, before any exchange, instead of waiting for each
other.  The device side (two ranks give exactly one GPU's results) is tests/test_gpu_ranks.py.
"""
import ctypes as C
import json
import os
import socket
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out: str) -> None:
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    from soltrace_b200 import parallel, scenes
    from soltrace_b200.lib import load

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    res = {}
    try:
        ex = parallel.RankExchange(device="cpu")
        u64 = C.POINTER(C.c_ulonglong)
        send = np.array([rank + 5, 100 * rank, 2 ** 40 + rank], dtype=np.uint64)
        recv = np.zeros(3 * world, dtype=np.uint64)
        res["ag_rc"] = ex.c_allgather(send.ctypes.data_as(u64), recv.ctypes.data_as(u64), 3, None)
        res["gathered"] = recv.tolist()
        buf = np.array([rank + 1, 7 * rank, 2 ** 41], dtype=np.uint64)
        res["sum_rc"] = ex.c_allreduce(buf.ctypes.data_as(u64), 3, parallel.OP_SUM, None)
        res["sum"] = buf.tolist()
        buf = np.array([rank + 1, 7 * rank, 2 ** 41 - rank], dtype=np.uint64)
        res["max_rc"] = ex.c_allreduce(buf.ctypes.data_as(u64), 3, parallel.OP_MAX, None)
        res["max"] = buf.tolist()
        api = load()
        ctx = api.st_create_context()
        scenes.push(api, ctx, scenes.dish_scene(100))
        res["bad_rank"] = api.st_b200_set_ranks(ctx, world, world, ex.c_allgather, ex.c_allreduce, None)
        res["no_callbacks"] = api.st_b200_set_ranks(ctx, rank, world, None, None, None)
        res["set"] = ex.attach(api, ctx)
        res["run"] = api.run(ctx, 1)  # no GPU here: fails on every rank before any exchange
        res["messages"] = api.messages(ctx)
        api.st_free_context(ctx)
        units, dev, wall = parallel.combine(1234.0, 10.0 + rank, 20.0 - rank, device="cpu")
        res["combine"] = [units, dev, wall]
        res["errors"] = ex.errors
    finally:
        dist.destroy_process_group()
    with open(out, "w") as fh:
        json.dump(res, fh)


def test_rank_exchange_two_gloo_ranks(tmp_path):
    world, port = 2, _free_port()
    outs = [str(tmp_path / f"rank{r}.json") for r in range(world)]
    procs = [subprocess.Popen([sys.executable, __file__, str(r), str(world), str(port), outs[r]])
             for r in range(world)]
    for p in procs:
        assert p.wait(timeout=180) == 0
    res = [json.load(open(o)) for o in outs]
    for r in res:
        assert (r["ag_rc"], r["sum_rc"], r["max_rc"]) == (1, 1, 1), r["errors"]
        assert r["gathered"] == [5, 0, 2 ** 40, 6, 100, 2 ** 40 + 1]  # rank-major
        assert r["sum"] == [3, 7, 2 ** 42]
        assert r["max"] == [2, 7, 2 ** 41]
        assert r["bad_rank"] == -1 and r["no_callbacks"] == -1 and r["set"] == 1
        assert r["run"] == -1 and any("CUDA" in m for m in r["messages"])
        assert r["combine"] == [1234.0, 11.0, 20.0]


def test_combine_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    from soltrace_b200 import parallel

    assert parallel.combine(5.0, 1.5, 2.5) == (5.0, 1.5, 2.5)


if __name__ == "__main__":
    _worker(int(sys.argv[1]), int(sys.argv[2]), int(sys.argv[3]), sys.argv[4])
