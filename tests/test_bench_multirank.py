"""The multi-process form of bench.py on CPU: two ranks over gloo (the GPU
runs use NCCL with the same calls).  Each rank is an independent replica;
the job's time is the largest rank's, and the aggregate counts every
rank's systems.  The reference arm prints only on rank 0."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RANK_SCRIPT = r"""
import json, sys
sys.path.insert(0, sys.argv[1])
import bench
rank, world, local, dist = bench.dist_setup(2, backend="gloo")
job = bench.max_over_ranks(1.5 + rank, dist, "cpu")
value = bench.aggregate_ns_per_day(100, 3, world, job)
dist.barrier()
print(json.dumps({"rank": rank, "world": world, "local": local, "job": job, "value": value}))
dist.destroy_process_group()
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_take_the_max_and_aggregate():
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE="2", LOCAL_RANK=str(r),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", RANK_SCRIPT, ROOT], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=120)
        assert p.returncode == 0, err[-2000:]
        outs.append(json.loads(out.strip().splitlines()[-1]))
    expect = 100 * 0.002e-3 * 3 * 2 / (2.5e-3) * 86400.0
    for r, o in enumerate(outs):
        assert o["rank"] == r and o["world"] == 2 and o["local"] == r
        assert o["job"] == 2.5
        assert abs(o["value"] - expect) < 1e-9 * expect


def test_reference_arm_prints_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "3"], env=env, capture_output=True, text=True,
                       timeout=120)
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.strip() == ""
