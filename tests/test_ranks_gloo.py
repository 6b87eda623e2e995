"""The multi-rank path of the batched scan on the CPU: two gloo ranks shard
the 64-instance draw, take the job time as the max over ranks and gather the
per-instance results -- the same helpers bench.py uses over NCCL."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out_dir):
    import datetime
    import json
    import torch.distributed as dist
    from nulattice_b200 import batch as B
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        inst = B.draw_instances(64, 0)
        mine = B.shard(inst, rank, world)
        local = [{"A": a, "L": l, "C2": c2, "C3": c3, "rank": rank} for a, l, c2, c3 in mine]
        load = sum(B.instance_cost(a, l) for a, l, _, _ in mine)
        t_job = B.max_over_ranks(1.0 + rank)
        all_res = B.gather_results(local)
        total_load = B.gather_results([load])
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"t_job": t_job, "n_local": len(local), "results": all_res, "loads": total_load}, f)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_reduce_and_gather(tmp_path):
    import json
    from nulattice_b200 import batch as B
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    outs = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(2)]
    inst = B.draw_instances(64, 0)
    for o in outs:
        assert o["t_job"] == 2.0                       # the slowest rank's time on both ranks
        assert len(o["results"]) == 64                  # every instance exactly once
        got = sorted((r["A"], r["L"], r["C2"], r["C3"]) for r in o["results"])
        assert got == sorted(tuple(x) for x in inst)
        # rank order of the gather, both ranks hold work, the loads are balanced
        ranks = [r["rank"] for r in o["results"]]
        assert ranks == sorted(ranks) and set(ranks) == {0, 1}
        assert max(o["loads"]) <= 1.25 * min(o["loads"])
    assert outs[0]["results"] == outs[1]["results"]
    assert outs[0]["n_local"] + outs[1]["n_local"] == 64


def test_helpers_without_a_process_group():
    from nulattice_b200 import batch as B
    assert B.max_over_ranks(3.5) == 3.5
    assert B.gather_results([1, 2]) == [1, 2]
