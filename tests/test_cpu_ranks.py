"""The replica plumbing of bench.py with world_size 2 on CPU (gloo):
barriers and the max-over-ranks of the timed region, and the reference arm
printing one line from rank 0 only. Rendezvous on 127.0.0.1."""
import json
import os
import re
import socket
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def torchrun(args, timeout=240):
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port())] + args
    env = dict(os.environ, OMP_NUM_THREADS="1", ORACLE_THREADS="2", CUDA_VISIBLE_DEVICES="")
    return subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=timeout)


def test_ranks_barrier_and_max_over_ranks(tmp_path):
    script = tmp_path / "ranks_probe.py"
    script.write_text(
        "import json, sys\n"
        f"sys.path.insert(0, {str(ROOT)!r})\n"
        "import bench\n"
        "r = bench.Ranks()\n"
        "r.init(timeout_s=60)\n"
        "r.barrier()\n"
        "m = r.max(1.5 + r.rank)\n"
        "r.barrier()\n"
        "print(json.dumps({'rank': r.rank, 'world': r.world, 'max': m}), flush=True)\n"
        "r.close()\n")
    res = torchrun([str(script)])
    assert res.returncode == 0, res.stderr[-2000:]
    # the two ranks share stdout: their lines may interleave, so pick out the objects
    lines = [json.loads(m) for m in re.findall(r"\{[^{}]*\}", res.stdout)]
    assert sorted(l["rank"] for l in lines) == [0, 1]
    assert all(l["world"] == 2 and l["max"] == 2.5 for l in lines)


def test_reference_arm_prints_one_line_from_rank_zero():
    res = torchrun(["bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3",
                    "--ref-n", "14"])
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [l for l in res.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] == "port" and d["unit"] == "s" and d["higher_is_better"] is False
