"""The N > 1 plumbing of bench.py, on CPU: two ranks as separate processes
(gloo backend, rendezvous on 127.0.0.1), as `torch.distributed.run` would
start them. The path has no exchange step, so N GPUs run N independent
replicas; what is shared is the barrier around the timed region, the
max-over-ranks device time and the whole-job throughput computed from it.
The reference arm runs on rank 0 alone."""
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import json, sys
sys.path.insert(0, sys.argv[1])
import bench
world, rank, local = bench.dist_setup(None)
bench.barrier(world)
ms = [12.5, 14.0][rank]                          # this rank's device time for the timed steps
ms_max = bench.max_over_ranks(ms, world)
value = bench.job_tflops(world, 10, 8.8e12, ms_max)
ref = bench.run_reference(None, world, rank, local) if rank != 0 else "rank0"
bench.barrier(world)
import torch.distributed as dist
dist.destroy_process_group()
print(json.dumps({"rank": rank, "world": world, "ms_max": ms_max, "value": value, "ref": ref}))
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_share_barrier_and_max_time():
    import json

    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", SCRIPT, ROOT], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=240)
        assert p.returncode == 0, err[-2000:]
        outs.append(json.loads(out.strip().splitlines()[-1]))
    for o in outs:
        assert o["world"] == 2
        assert o["ms_max"] == 14.0                      # the slowest rank's time
        # 2 replicas x 10 steps x 8.8e12 flops in 14 ms
        assert abs(o["value"] - 2 * 10 * 8.8e12 / 14e-3 / 1e12) < 1e-9
    assert outs[1]["ref"] is None                        # only rank 0 runs the reference arm
