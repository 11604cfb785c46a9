"""The N > 1 path of bench.py on CPU: two `gloo` ranks.

The factorization does not shard across GPUs here: `bench.py --gpus N` runs N
replicas, each factoring and solving its own operator (per-rank seeds), and the
only collectives are the barrier and the max over ranks of the step times. This
test runs that host logic with world_size 2 on the gloo backend: each rank
reports a different step time, both must get the slowest one, the whole-job
value must count both replicas, and the replicas' operators must differ.
"""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RANK_SCRIPT = r"""
import datetime, json, os, sys
import numpy as np
import torch.distributed as dist
sys.path.insert(0, os.environ["HIF_ROOT"])
import bench
from hifde3d_b200 import synth

rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
try:
    ms = [700.0, 1300.0][rank]
    e2e = [0.9, 1.6][rank]
    dist.barrier()
    ms_max, e2e_max = bench.replica_times(ms, e2e, world)
    seed_op, seed_rhs = bench.replica_seeds(rank)
    ax, _, _ = synth.face_coefficients_grf(7, seed_op, 1.0 / 16, 1.0)
    b = synth.dof_vector(7, seed_rhs)
    print(json.dumps({"rank": rank, "ms": ms_max, "e2e": e2e_max,
                      "value": bench.job_value(world, ms_max),
                      "a_sum": float(np.sum(ax)), "b_sum": float(np.sum(b))}))
finally:
    dist.destroy_process_group()
"""


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_replicas_take_the_slowest_rank():
    pytest.importorskip("torch")
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), HIF_ROOT=ROOT,
                   CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", RANK_SCRIPT], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                      text=True))
    outs = []
    for p in procs:
        try:
            out, err = p.communicate(timeout=240)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
        assert p.returncode == 0, err[-2000:]
        outs.append(json.loads(out.strip().splitlines()[-1]))
    outs.sort(key=lambda r: r["rank"])
    for r in outs:
        assert r["ms"] == 1300.0
        assert r["e2e"] == 1.6
        assert np.isclose(r["value"], 2 * 1e3 / 1300.0)
    # different operators and right-hand sides per replica
    assert outs[0]["a_sum"] != outs[1]["a_sum"]
    assert outs[0]["b_sum"] != outs[1]["b_sum"]


def test_single_rank_needs_no_process_group():
    import bench

    assert bench.replica_times(5.0, 0.2, 1) == (5.0, 0.2)
    assert bench.job_value(1, 500.0) == 2.0
    assert bench.replica_seeds(0) == (2, 0)
