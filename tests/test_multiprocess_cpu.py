"""The N > 1 plumbing of bench.py on CPU: two gloo ranks, each an
independent replica (no data-path collective), timing reduced as the max over
ranks; and the reference arm printing from rank 0 only."""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]

WORKER = r"""
import os, sys, json
sys.path.insert(0, sys.argv[1])
import bench
import torch.distributed as dist
class A: impl = "reference"
world, rank, local = bench.dist_init(A)
assert dist.get_backend() == "gloo"
bench.barrier(world)
t = bench.allreduce_max(world, 1.0 + rank)
print(json.dumps({"rank": rank, "world": world, "max": t}))
dist.destroy_process_group()
"""


def _spawn(nproc, script_args, env_extra=None, timeout=120):
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(29500 + os.getpid() % 1000),
               WORLD_SIZE=str(nproc))
    env.update(env_extra or {})
    procs = []
    for r in range(nproc):
        e = dict(env, RANK=str(r), LOCAL_RANK=str(r))
        procs.append(subprocess.Popen([sys.executable, *script_args], env=e, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=timeout)
        assert p.returncode == 0, err[-2000:]
        outs.append(out)
    return outs


def test_two_gloo_ranks_reduce_max(tmp_path):
    script = tmp_path / "worker.py"
    script.write_text(WORKER)
    outs = _spawn(2, [str(script), str(ROOT)])
    res = [json.loads(o.strip().splitlines()[-1]) for o in outs]
    assert sorted(r["rank"] for r in res) == [0, 1]
    assert all(r["world"] == 2 and r["max"] == 2.0 for r in res)


@pytest.mark.skipif(not any((ROOT / "oracle" / "_ref").glob("olb_ref_simd_q19_f32_*")),
                    reason="reference SIMD driver not built")
def test_reference_arm_prints_once_under_two_ranks():
    outs = _spawn(2, [str(ROOT / "bench.py"), "--impl", "reference", "--n", "24", "--steps", "3",
                      "--warmup", "1"], env_extra={"OMP_NUM_THREADS": "2"}, timeout=300)
    lines = [l for o in outs for l in o.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference" and rec["n_gpus"] == 2 and rec["value"] > 0
    assert rec["cpu_baseline"]["kind"] == "reference"
