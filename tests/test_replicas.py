"""CPU: the multi-process plumbing of `bench.py --gpus N` (replicas: one
process per GPU, independent channels, no data-path collective) on two
`gloo` ranks.

The ranks meet only at the barriers around the timed region and in the
maximum of their times; each replica steps its own seeded state (a different
seed per rank), and for the ensemble workload each rank holds a full ensemble
of the same shapes with its own seeds.  Under torchrun the reference arm runs
on rank 0 alone, and the other ranks exit 0 without output.
"""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

import bench

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    r, w, local, dist = bench.init_ranks("gloo", timeout_s=60)
    barrier, max_over_ranks = bench.rank_ops(dist, "cpu")
    barrier()
    m = max_over_ranks(1.5 + r)
    members = bench.ensemble_members(bench.CONFIGS["c4"], r)
    out.put((r, w, local, m, [mm[:3] for mm in members], [mm[5] for mm in members]))
    bench.finish_ranks(dist)


def test_two_gloo_ranks_share_only_timing():
    world, port = 2, free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, w0, l0, m0, shapes0, seeds0), (r1, w1, l1, m1, shapes1, seeds1) = got
    assert (r0, r1, w0, w1, l0, l1) == (0, 1, 2, 2, 0, 1)
    # the timing every rank reports is the slowest rank's
    assert m0 == m1 == 2.5
    # weak scaling: the same ensemble shapes on every rank, independent seeds
    assert shapes0 == shapes1 and len(shapes0) == 256
    assert not set(seeds0) & set(seeds1)


def test_single_rank_needs_no_process_group():
    r, w, local, dist = bench.init_ranks("gloo")
    assert (w, dist) == (1, None)
    barrier, max_over_ranks = bench.rank_ops(dist, "cpu")
    barrier()
    assert max_over_ranks(3.25) == 3.25


def test_reference_arm_runs_on_rank_zero_only():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), "bench.py", "--impl", "reference",
           "--gpus", "2", "--config", "c1", "--steps", "1", "--warmup", "0"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
