"""The QAOA sweep split across ranks (aleph_b200/sweep.py), on CPU.

The partition is contiguous and balanced by sum(2^n); with world_size 2 over
gloo each rank evaluates its share (here with the oracle: the GPU sweep kernel
needs a device) and the all-gather rebuilds the same <C> vector that one rank
computes alone. Multi-GPU runs of the sweep are unmeasured on hardware: every
run available here has one GPU.
"""
import json
import re

import numpy as np
import pytest

from aleph_b200.sweep import partition_by_work
from tests.test_cpu_ranks import ROOT, torchrun


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_partition_is_contiguous_and_balanced(world):
    rng = np.random.default_rng(world)
    sizes = [int(x) for x in rng.integers(12, 25, 4096)]
    parts = partition_by_work(sizes, world)
    assert parts[0][0] == 0 and parts[-1][1] == len(sizes)
    assert all(parts[r][1] == parts[r + 1][0] for r in range(world - 1))
    work = [sum(1 << sizes[i] for i in range(a, b)) for a, b in parts]
    ideal = sum(work) / world
    assert max(work) - ideal <= (1 << max(sizes))  # off by at most one set


def test_partition_with_fewer_sets_than_ranks():
    parts = partition_by_work([5, 7], 4)
    covered = [i for a, b in parts for i in range(a, b)]
    assert covered == [0, 1]


SCRIPT = """
import json, sys
sys.path.insert(0, {root!r})
import numpy as np
import bench
from aleph_b200 import workloads
from aleph_b200.sweep import sharded_sweep
from oracle import oracle

def evaluate(graphs, gam, bet):
    out = []
    for (n, e), g, b in zip(graphs, gam, bet):
        psi, _ = oracle.run(n, workloads.qaoa_maxcut(n, e, g, b).instructions)
        out.append(sum(0.5 * (1 - oracle.expectation(psi, [(i, "Z"), (j, "Z")])) for i, j in e))
    return np.array(out)

rng = np.random.default_rng(3)
graphs = []
for n in rng.integers(4, 10, 24):
    n = int(n)
    e = sorted({{(int(min(i, j)), int(max(i, j))) for i, j in rng.integers(0, n, (n + 2, 2)) if i != j}})
    graphs.append((n, e))
gam = rng.uniform(0, np.pi, (24, 2))
bet = rng.uniform(0, np.pi, (24, 2))
r = bench.Ranks()
r.init(timeout_s=60)
full = sharded_sweep(graphs, gam, bet, evaluate, r.rank, r.world)
alone = evaluate(graphs, gam, bet)
print(json.dumps({{"rank": r.rank, "full": full.tolist(), "alone": alone.tolist()}}), flush=True)
r.close()
"""


def test_two_ranks_gather_the_single_rank_vector(tmp_path):
    script = tmp_path / "sweep_probe.py"
    script.write_text(SCRIPT.format(root=str(ROOT)))
    res = torchrun([str(script)])
    assert res.returncode == 0, res.stderr[-2000:]
    # the ranks share one stdout, so two lines can arrive run together: decode
    # each object from where it starts
    dec = json.JSONDecoder()
    lines = [dec.raw_decode(res.stdout, m.start())[0] for m in re.finditer(r"\{\"rank\"", res.stdout)]
    assert sorted(l["rank"] for l in lines) == [0, 1]
    for l in lines:
        assert l["full"] == l["alone"]  # identical doubles: same evaluation, gathered


# ---- the learned planner's training-data collection, split across ranks ----------------
def test_training_circuits_shard_covers_every_circuit_once():
    from aleph_b200 import learned

    circuits = learned.training_circuits()
    for world in (1, 2, 3, 8):
        parts = [learned.shard_circuits(circuits, r, world) for r in range(world)]
        ids = sorted(id(c) for p in parts for c in p)
        assert ids == sorted(id(c) for c in circuits)
        loads = [sum(learned.circuit_work(n, i) for n, i in p) for p in parts]
        biggest = max(learned.circuit_work(n, i) for n, i in circuits)
        assert max(loads) - min(loads) <= biggest  # largest-first, least-loaded rank


COLLECT_SCRIPT = """
import json, sys
sys.path.insert(0, {root!r})
import numpy as np
import torch.distributed as dist
from aleph_b200 import learned

dist.init_process_group("gloo")
rank, world = dist.get_rank(), dist.get_world_size()
circuits = learned.training_circuits(sizes=(10, 12))
mine = learned.shard_circuits(circuits, rank, world)
# stand-in for the per-pass samples a GPU run records: one row per circuit
X = np.array([[n, len(i)] for n, i in mine], np.float32).reshape(-1, 2)
y = np.array([float(n * 1000 + len(i)) for n, i in mine], np.float32)
Xa, ya = learned.gather_samples(X, y, world)
print(json.dumps({{"rank": rank, "y": sorted(ya.tolist()), "rows": int(Xa.shape[0])}}), flush=True)
dist.destroy_process_group()
"""


def test_training_samples_gather_over_two_ranks(tmp_path):
    from aleph_b200 import learned

    script = tmp_path / "collect_probe.py"
    script.write_text(COLLECT_SCRIPT.format(root=str(ROOT)))
    res = torchrun([str(script)])
    assert res.returncode == 0, res.stderr[-2000:]
    dec = json.JSONDecoder()
    lines = [dec.raw_decode(res.stdout, m.start())[0] for m in re.finditer(r"\{\"rank\"", res.stdout)]
    assert sorted(l["rank"] for l in lines) == [0, 1]
    want = sorted(float(n * 1000 + len(i)) for n, i in learned.training_circuits(sizes=(10, 12)))
    for l in lines:
        assert l["y"] == want and l["rows"] == len(want)
