"""Multi-rank logic of the weakly scaled trace, as two gloo ranks on the CPU.

`soltrace_b200.parallel.combine` is what bench.py runs after the timed steps on every
rank (over NCCL on the GPU box): units summed, device and wall times max over ranks,
receiver flux maps summed.  Here two processes run it over gloo with known per-rank
inputs; the test checks the totals on both ranks, and that the ranks' seeds differ.
"""
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


def _rank_inputs(rank: int):
    rng = np.random.default_rng(100 + rank)
    flux = rng.integers(0, 1000, size=(4, 5)).astype(np.int64)
    return 1000.0 * (rank + 1), 10.0 + rank, 20.0 - rank, flux


def _worker(rank: int, world: int, port: int, out: str) -> None:
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    from soltrace_b200 import parallel

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        units, dev, wall, flux = _rank_inputs(rank)
        u, d, w, f = parallel.combine(units, dev, wall, flux, device="cpu")
        with open(out, "w") as fh:
            json.dump({"units": u, "dev": d, "wall": w, "flux": f.tolist(),
                       "seed": parallel.rank_seed(3, rank)}, fh)
    finally:
        dist.destroy_process_group()


def test_combine_two_gloo_ranks(tmp_path):
    world, port = 2, _free_port()
    outs = [str(tmp_path / f"rank{r}.json") for r in range(world)]
    procs = [subprocess.Popen([sys.executable, __file__, str(r), str(world), str(port), outs[r]])
             for r in range(world)]
    for p in procs:
        assert p.wait(timeout=120) == 0
    res = [json.load(open(o)) for o in outs]
    inputs = [_rank_inputs(r) for r in range(world)]
    want_flux = sum(i[3] for i in inputs)
    for r in res:
        assert r["units"] == sum(i[0] for i in inputs)
        assert r["dev"] == max(i[1] for i in inputs)
        assert r["wall"] == max(i[2] for i in inputs)
        np.testing.assert_array_equal(np.array(r["flux"]), want_flux)
    assert res[0]["seed"] != res[1]["seed"]


def test_combine_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    from soltrace_b200 import parallel

    flux = np.arange(6, dtype=np.int64).reshape(2, 3)
    u, d, w, f = parallel.combine(5.0, 1.5, 2.5, flux)
    assert (u, d, w) == (5.0, 1.5, 2.5)
    np.testing.assert_array_equal(f, flux)


if __name__ == "__main__":
    _worker(int(sys.argv[1]), int(sys.argv[2]), int(sys.argv[3]), sys.argv[4])
