"""A run split over ranks (st_b200_set_ranks) gives exactly the single-GPU run.

Two and three rank processes (gloo for the exchanges, all on the one GPU this test has:
their kernels never wait on one another, the ranks meet only on the host between launches)
trace the 300-heliostat field with records on.  Against the same st_sim_run in this process
without ranks: SunRayCount, hits, stage entries and intersections, the receiver flux map and
every stage's per-element counts must be equal on every rank, and the ranks' records
together must be the single run's records (same rays, same ray numbers, same positions bit
for bit).  The sun-ray range of every batch is split contiguously over the ranks, each ray
keeping its own random stream, which is what makes the results independent of the rank count.
"""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
MAP = (2, 1, 1, 72, 40, 0.0, 4.0, -5.0, 5.0, 1)
HITS, SEED = 20000, 23

pytestmark = pytest.mark.gpu


def _scene():
    sys.path.insert(0, ROOT)
    from soltrace_b200 import scenes
    return scenes.field_scene(300, HITS, dynamic_group=False)


def _trace(api, ctx, prec):
    from soltrace_b200 import scenes
    sc = _scene()
    scenes.push(api, ctx, sc)
    api.st_b200_set_precision(ctx, prec)
    api.st_b200_add_flux_map(ctx, *MAP)
    n = api.run(ctx, SEED)
    assert n > 0, api.messages(ctx)
    st = api.stats(ctx)
    out = {"n": n, "records": api.records(ctx), "flux": api.flux(ctx, 0, MAP[3], MAP[4]),
           "stats": {k: st[k] for k in ("sun_rays", "ray_hits", "ray_stage_units", "intersections")},
           "entries": st["stage_entries"][:2],
           "counts": [np.stack(api.element_counts(ctx, s + 1, len(stg.elements))) for s, stg in enumerate(sc.stages)]}
    return out


def _worker(rank, world, port, prec, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, HERE)
    from soltrace_b200 import parallel
    from soltrace_b200.lib import load

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        api = load()
        ex = parallel.RankExchange(device="cpu")
        ctx = api.st_create_context()
        assert ex.attach(api, ctx) == 1
        r = _trace(api, ctx, prec)
        api.st_free_context(ctx)
        np.savez(out, flux=r["flux"], entries=np.array(r["entries"]), counts=np.concatenate(r["counts"], axis=1),
                 **{"rec_" + k: v for k, v in r["records"].items()})
        with open(out + ".json", "w") as fh:
            json.dump({"stats": r["stats"], "errors": ex.errors}, fh)
    finally:
        dist.destroy_process_group()


def _sorted(rec):
    order = np.lexsort((np.arange(len(rec["raynum"])), rec["raynum"], rec["stage"]))
    return {k: np.asarray(v)[order] for k, v in rec.items()}


@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "mixed"])
@pytest.mark.parametrize("world", [2, 3])
def test_ranks_equal_single_gpu_run(product, tmp_path, world, prec):
    ctx = product.st_create_context()
    try:
        one = _trace(product, ctx, prec)
    finally:
        product.st_free_context(ctx)
    port = _free_port()
    outs = [str(tmp_path / f"rank{r}.npz") for r in range(world)]
    env = dict(os.environ, NCCL_NVLS_ENABLE="0")
    procs = [subprocess.Popen([sys.executable, __file__, str(r), str(world), str(port), str(prec), outs[r]], env=env)
             for r in range(world)]
    for p in procs:
        assert p.wait(timeout=300) == 0
    recs = []
    for o in outs:
        d = np.load(o)
        meta = json.load(open(o + ".json"))
        assert not meta["errors"]
        assert meta["stats"] == one["stats"]
        np.testing.assert_array_equal(d["flux"], one["flux"])
        assert d["entries"].tolist() == list(one["entries"])
        np.testing.assert_array_equal(d["counts"], np.concatenate(one["counts"], axis=1))
        recs.append({k[4:]: d[k] for k in d.files if k.startswith("rec_")})
    assert all(len(r["x"]) > 0 for r in recs)  # every rank traced part of the run
    merged = {k: np.concatenate([r[k] for r in recs]) for k in recs[0]}
    a, b = _sorted(merged), _sorted(one["records"])
    for k in b:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


if __name__ == "__main__":
    _worker(int(sys.argv[1]), int(sys.argv[2]), int(sys.argv[3]), int(sys.argv[4]), sys.argv[5])
