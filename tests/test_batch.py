"""Batched boxes: the workload generator, the longest-processing-time shard of boxes over
ranks (checked with two gloo ranks on CPU), and on a GPU the batch path against single
contexts."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from apcloud import ics


def test_batch_boxes_recipe():
    boxes = ics.batch_boxes()
    assert len(boxes) == 96
    assert {b.n for b in boxes} <= {s ** 3 for s in ics.BATCH_SIDES}
    assert sum(b.kind == "ball" for b in boxes) == 48
    assert all(0.15 <= b.radius <= 0.35 for b in boxes if b.kind == "ball")
    assert all(0.1 <= b.rms_spacing <= 0.3 for b in boxes if b.kind == "zeldovich")
    assert all((b.a_start, b.a_end, b.steps, b.omega0) == (0.05, 0.5, 32, 1.0) for b in boxes)
    assert len({b.seed for b in boxes}) == 96
    again = ics.batch_boxes()
    assert [(b.n, b.seed, b.gfd_c) for b in boxes] == [(b.n, b.seed, b.gfd_c) for b in again]


@pytest.mark.parametrize("parts", [1, 2, 3, 8])
def test_lpt_partition_covers_and_balances(parts):
    costs = [b.n * b.steps for b in ics.batch_boxes()]
    bins = ics.lpt_partition(costs, parts)
    flat = sorted(i for b in bins for i in b)
    assert flat == list(range(len(costs)))
    loads = [sum(costs[i] for i in b) for b in bins]
    # LPT bound: no bin exceeds the mean by more than the largest item
    assert max(loads) <= sum(costs) / parts + max(costs)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, ws: int, port: int, out_dir: str):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(ws), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import json

    import bench

    d = bench.Dist(0, backend="gloo")
    cfgs = ics.batch_boxes()
    mine = bench.batch_shard(cfgs, ws, rank)
    work = float(sum(cfgs[i].n * cfgs[i].steps for i in mine))
    import torch.distributed as td

    gathered = [None] * ws
    td.all_gather_object(gathered, mine)
    res = {"mine": mine, "all": gathered, "max": d.max(work), "sum": d.sum(work)}
    d.barrier()
    d.close()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump(res, f)


def test_batch_shard_two_gloo_ranks(tmp_path):
    import json

    import torch.multiprocessing as mp

    ws = 2
    mp.start_processes(_rank_main, args=(ws, _free_port(), str(tmp_path)), nprocs=ws, start_method="spawn",
                       join=True)
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(ws)]
    cfgs = ics.batch_boxes()
    costs = [c.n * c.steps for c in cfgs]
    assert res[0]["all"] == res[1]["all"]
    assert sorted(res[0]["mine"] + res[1]["mine"]) == list(range(len(cfgs)))
    assert not set(res[0]["mine"]) & set(res[1]["mine"])
    loads = [sum(costs[i] for i in r["mine"]) for r in res]
    assert res[0]["max"] == res[1]["max"] == max(loads)
    assert res[0]["sum"] == sum(costs)


@pytest.mark.gpu
@pytest.mark.parametrize("workers", [1, 4])
def test_batch_matches_single_contexts(workers):
    """Boxes stepped together through apc_batch_step end exactly where the same boxes end
    when each runs alone through its own context: with one host thread running all six
    boxes as fibers, and with four threads."""
    from apcloud import binding
    from apcloud.batch import BatchRun
    from apcloud.controller import Controller

    cfgs = ics.batch_boxes(n_boxes=12, seed=11, sides=(16, 24))[:6]
    steps = 3
    br = BatchRun(cfgs, precision=binding.APC_PREC_MIXED, n_workers=workers)
    br.start()
    for _ in range(steps):
        br.step()
    got = [np.stack(g.particles()) for g in br.path.boxes]
    br.close()
    for c, arr in zip(cfgs, got):
        g = binding.GpuPath(c.particles(), c.depth, c.gfd_c, c.lm, restart=c.restart, rtol=c.rtol,
                            precision=binding.APC_PREC_MIXED)
        ctl = Controller(g, c.n, c.omega0, c.omegal, c.a_start, c.a_end, c.delta_a)
        ctl.start()
        for _ in range(steps):
            ctl.step()
        ref = np.stack(g.particles())
        g.close()
        assert np.array_equal(arr, ref), c.name


@pytest.mark.gpu
def test_queued_batch_solves_match_single_contexts():
    """APC_BATCH_SOLVE_QUEUED: every box's density solve, then every potential solve, run in
    one cooperative launch whose block groups take boxes from a device work queue.  Each
    box meets the same stopping test as alone, with its sums over other block counts, so
    the bar is the solver's accuracy: accelerations within 1e-6 RMS (the force-error bound)
    and positions within 1e-8 of the box after three steps, every box converged.  Two
    solutions that both meet rtol 1e-10 differ by up to cond(A) 1e-10, about 1e-8 in the
    accelerations of these boxes; the persistent body and the graph kernels also split
    their row sums over different lane counts."""
    from apcloud import binding
    from apcloud.batch import BatchRun
    from apcloud.controller import Controller

    cfgs = ics.batch_boxes(n_boxes=12, seed=11, sides=(16, 24, 32))[:8]
    steps = 3
    br = BatchRun(cfgs, precision=binding.APC_PREC_MIXED, n_workers=4, solve_mode=binding.APC_BATCH_SOLVE_QUEUED)
    br.start()
    for _ in range(steps):
        br.step()
    assert br.path.solve_ms() > 0.0
    got = [(np.stack(g.particles()), g.solve_stats()) for g in br.path.boxes]
    br.close()
    for c, (arr, st) in zip(cfgs, got):
        assert st["density_reason"] == 2 and st["potential_reason"] == 2, (c.name, st)
        g = binding.GpuPath(c.particles(), c.depth, c.gfd_c, c.lm, restart=c.restart, rtol=c.rtol,
                            precision=binding.APC_PREC_MIXED)
        ctl = Controller(g, c.n, c.omega0, c.omegal, c.a_start, c.a_end, c.delta_a)
        ctl.start()
        for _ in range(steps):
            ctl.step()
        ref = np.stack(g.particles())
        g.close()
        d = arr[:3] - ref[:3]
        d -= np.round(d)
        assert np.max(np.abs(d)) <= 1e-8, c.name
        a, b = arr[6:9], ref[6:9]
        rms = float(np.sqrt(np.mean(np.sum((a - b) ** 2, 0)) / np.mean(np.sum(b ** 2, 0))))
        assert rms <= 1e-6, (c.name, rms)
