"""Amplitude sharding (aleph_b200/dist.py) on CPU: the router, the per-rank
specialisation and the exchange, with numpy rank slices and the oracle as
each rank's executor, against the single-node oracle at 1e-12. One test runs
every rank in this process (in-process exchanges); the others run 2 and 4
gloo processes (exchanges over torch.distributed), as the reference's CPU
reference executor does for its planner (crates/aleph-sv/src/dist_ref.rs).
The multi-GPU transport (NCCL) is unmeasured on hardware: every run here
has one GPU.
"""
import json
import os
import re
import subprocess
import sys

import numpy as np
import pytest

from aleph_b200 import circuit as C
from aleph_b200 import dist, workloads
from oracle import oracle
from tests.circuit_gen import random_circuit
from tests.test_cpu_ranks import ROOT, free_port

TOL = 1e-12


class NumpyRanks:
    """Rank slices as numpy arrays, each run by the oracle (test executor)."""

    def __init__(self, layout, ranks):
        self.layout, self.ranks = layout, list(ranks)
        self.slices = {r: np.zeros(1 << layout.m, dtype=np.complex128) for r in self.ranks}
        if 0 in self.slices:
            self.slices[0][0] = 1.0

    def bytes_view(self, r):
        import torch

        return torch.from_numpy(self.slices[r].view(np.uint8))

    def apply(self, r, instrs):
        if instrs:
            psi, _ = oracle.run(self.layout.m, instrs, state=self.slices[r])
            self.slices[r][:] = psi

    def statevector(self, r):
        return self.slices[r]

    def norm_sqr(self, r):
        return float(np.vdot(self.slices[r], self.slices[r]).real)


def run_numpy(circ, g, chunk=1 << 10):
    layout = dist.DistLayout(circ.num_qubits, g)
    plan = dist.plan_dist(circ.instructions, layout)
    ranks = NumpyRanks(layout, range(layout.ranks))
    st = dist.execute(plan, ranks, dist.Exchange(chunk_bytes=chunk))
    return dist.gather_statevector(st), plan


def phase_circuit(n, seed):
    rng = np.random.default_rng(seed)
    c = workloads.brickwall(n, 2, seed=seed)
    terms = [C.PhaseTerm(tuple(int(x) for x in rng.integers(1, 1 << n, size=int(rng.integers(0, 3)))),
                         float(rng.uniform(-3, 3))) for _ in range(10)]
    c.instructions.append(C.DiagonalPhase(n, terms))
    c.instructions.extend(workloads.brickwall(n, 2, seed=seed + 1).instructions)
    return c


CASES = {
    "random9": (lambda: random_circuit(9, 200, seed=71), (1, 2, 3)),
    "random10": (lambda: random_circuit(10, 160, seed=72), (2, 4)),
    "brickwall": (lambda: workloads.brickwall(10, 10, seed=73), (1, 3)),
    "qft": (lambda: workloads.qft_product(9, seed=74), (2, 3)),
    "grover": (lambda: workloads.grover(4, 11, 2), (2,)),
    "phase": (lambda: phase_circuit(9, 75), (1, 3)),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_sharded_run_matches_single_node(name):
    make, gs = CASES[name]
    c = make()
    c = C.Circuit(max(c.num_qubits, 6), c.instructions)
    want, _ = oracle.run(c.num_qubits, c.instructions)
    for g in gs:
        got, plan = run_numpy(c, g)
        assert np.abs(got - want).max() <= TOL, (name, g)


def test_router_keeps_nondiagonal_work_local():
    c = random_circuit(10, 300, seed=5)
    for g in (1, 3, 5):
        layout = dist.DistLayout(10, g)
        plan = dist.plan_dist(c.instructions, layout)
        assert sorted(plan.final_map) == list(range(10))
        for step in plan.steps:
            if isinstance(step, dist.LocalStep):
                for inst in step.instructions:
                    assert all(q < layout.m for q in dist.nondiagonal_targets(inst))
            else:
                assert layout.m <= step.global_qubit < 10


def test_diagonal_work_on_global_qubits_needs_no_exchange():
    # a brickwall's CZs and a QFT-like phase ladder touching the global qubits
    # are specialised per rank; only the one-qubit gates on global qubits move data
    n, g = 10, 2
    c = C.Circuit(n)
    for q in range(n - 1):
        c.add(C.Cz(), [q, q + 1]).add(C.CRz(0.3 * q), [q, n - 1]).add(C.Phase(0.2), [n - 2], [q])
    plan = dist.plan_dist(c.instructions, dist.DistLayout(n, g))
    assert plan.exchanges() == 0
    c.add(C.H(), [n - 1])
    assert dist.plan_dist(c.instructions, dist.DistLayout(n, g)).exchanges() == 1


def test_unsupported_instructions_and_layouts():
    with pytest.raises(dist.DistError):
        dist.DistLayout(4, 4)
    c = C.Circuit(6).add(C.H(), [0])
    c.measure(0, 0)
    with pytest.raises(dist.DistError):
        dist.plan_dist(c.instructions, dist.DistLayout(6, 1))
    wide = C.Circuit(6).add(C.UnitaryKq(np.eye(32)), [0, 1, 2, 3, 4])
    with pytest.raises(dist.DistError):  # 5 qubits do not fit 3 local ones
        dist.plan_dist(wide.instructions, dist.DistLayout(6, 3))


SCRIPT = """
import json, sys
sys.path.insert(0, {root!r})
import numpy as np
import torch.distributed as dist_
from aleph_b200 import dist, workloads
from tests.circuit_gen import random_circuit
from tests.test_cpu_dist import NumpyRanks

dist_.init_process_group("gloo")
rank, world = dist_.get_rank(), dist_.get_world_size()
c = random_circuit(10, 220, seed=81)
c.instructions.extend(workloads.qft_product(10, seed=82).instructions)
layout = dist.DistLayout(10, {g})
per = layout.ranks // world
plan = dist.plan_dist(c.instructions, layout)
ranks = NumpyRanks(layout, range(rank * per, (rank + 1) * per))
st = dist.execute(plan, ranks, dist.Exchange(chunk_bytes=1 << 9, world=world, rank=rank))
norm = dist.norm_sqr(st)
slices = [None] * world
dist_.all_gather_object(slices, {{r: ranks.slices[r] for r in ranks.ranks}})
if rank == 0:
    phys = np.concatenate([s[r] for s in slices for r in sorted(s)])
    got = dist.unmap(phys, plan.final_map)
    np.save({out!r}, got)
    print(json.dumps({{"norm": norm, "exchanges": plan.exchanges()}}), flush=True)
dist_.destroy_process_group()
"""


@pytest.mark.parametrize("world,g", [(2, 1), (2, 2), (4, 2), (4, 3)])
def test_sharded_run_over_gloo_processes(tmp_path, world, g):
    out = tmp_path / "state.npy"
    script = tmp_path / "dist_probe.py"
    script.write_text(SCRIPT.format(root=str(ROOT), g=g, out=str(out)))
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={world}",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), str(script)]
    env = dict(os.environ, OMP_NUM_THREADS="1", ORACLE_THREADS="1", CUDA_VISIBLE_DEVICES="")
    res = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr[-3000:]
    info = json.loads(re.findall(r"\{[^{}]*\}", res.stdout)[0])
    assert info["exchanges"] > 0 and abs(info["norm"] - 1.0) <= 1e-12
    c = random_circuit(10, 220, seed=81)
    c.instructions.extend(workloads.qft_product(10, seed=82).instructions)
    want, _ = oracle.run(10, c.instructions)
    assert np.abs(np.load(out) - want).max() <= TOL
