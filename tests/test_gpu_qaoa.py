"""Batched QAOA Max-Cut sweep (aleph_b200_qaoa_sweep) against the oracle.

Each set's reference value is the oracle's FP64 gate-by-gate run of the
build_qaoa circuit (crates/aleph-ir/src/ansatz.rs:71-98) followed by
<C> = sum_edges 1/2 (1 - <Z_i Z_j>) (ansatz.rs:100-117). Tolerances: FP64
state 1e-9 absolute; FP32 state 2e-5 relative (FP32 tolerance class, with
<C> reduced in FP64).
"""
import numpy as np
import pytest

from aleph_b200 import workloads
from aleph_b200.backend import (B200SvBackend, DuplicateQubit, NonFiniteParam, QubitOutOfRange,
                                TooManyQubits)
from oracle import oracle

pytestmark = pytest.mark.gpu


def random_graph(n, rng):
    if n % 2 == 0 and n >= 4:
        return workloads.random_3_regular(n, rng)
    edges = set()
    while len(edges) < (3 * n) // 2:
        i, j = (int(x) for x in rng.choice(n, 2, replace=False))
        edges.add((min(i, j), max(i, j)))
    return sorted(edges)


def oracle_cost(n, edges, gammas, betas):
    psi, _ = oracle.run(n, workloads.qaoa_maxcut(n, edges, gammas, betas).instructions)
    return sum(0.5 * (1.0 - oracle.expectation(psi, [(i, "Z"), (j, "Z")])) for (i, j) in edges)


def make_batch(sizes, p, seed):
    rng = np.random.default_rng(seed)
    graphs = [(n, random_graph(n, rng)) for n in sizes]
    gam = rng.uniform(0, np.pi, (len(sizes), p))
    bet = rng.uniform(0, np.pi, (len(sizes), p))
    return graphs, gam, bet


@pytest.mark.parametrize("precision,tol", [("f64", 1e-9), ("f32", 2e-5)])
def test_sweep_matches_oracle_smem_and_streamed(precision, tol):
    # n <= 13 (f64) / 14 (f32) stay in shared memory; larger ones are streamed
    sizes = [4, 7, 12, 13, 14, 15, 16, 17, 12, 16]
    graphs, gam, bet = make_batch(sizes, 3, seed=5)
    be = B200SvBackend(seed=0, precision=precision)
    got = be.qaoa_sweep(graphs, gam, bet)
    for k, (n, edges) in enumerate(graphs):
        want = oracle_cost(n, edges, gam[k], bet[k])
        err = abs(got[k] - want) if precision == "f64" else abs(got[k] - want) / max(1.0, abs(want))
        assert err <= tol, (k, n, got[k], want)


def test_sweep_graph_replay_with_new_angles_and_new_layout():
    be = B200SvBackend(seed=0, precision="f64")
    graphs, gam, bet = make_batch([10, 14, 15], 2, seed=6)
    first = be.qaoa_sweep(graphs, gam, bet)
    gam2, bet2 = gam[::-1].copy(), bet * 0.5
    second = be.qaoa_sweep(graphs, gam2, bet2)  # same layout: graph replay with new inputs
    for k, (n, edges) in enumerate(graphs):
        assert abs(first[k] - oracle_cost(n, edges, gam[k], bet[k])) <= 1e-9
        assert abs(second[k] - oracle_cost(n, edges, gam2[k], bet2[k])) <= 1e-9
    graphs3, gam3, bet3 = make_batch([6, 9], 4, seed=7)  # new layout: recaptured
    third = be.qaoa_sweep(graphs3, gam3, bet3)
    for k, (n, edges) in enumerate(graphs3):
        assert abs(third[k] - oracle_cost(n, edges, gam3[k], bet3[k])) <= 1e-9


def test_sweep_single_edge_numpy():
    # independent dense check: |++>, exp(-i g Z(x)Z), Rx(2b)(x)Rx(2b), <C> = 1/2 (1 - <ZZ>)
    be = B200SvBackend(seed=0, precision="f64")
    g, b = 0.37, 1.21
    got = be.qaoa_sweep([(2, [(0, 1)])], [[g]], [[b]])[0]
    zz = np.array([1, -1, -1, 1], dtype=float)
    psi = np.full(4, 0.5, dtype=complex) * np.exp(-1j * g * zz)
    rx = np.array([[np.cos(b), -1j * np.sin(b)], [-1j * np.sin(b), np.cos(b)]])
    psi = np.kron(rx, rx) @ psi
    assert abs(got - 0.5 * (1 - np.vdot(psi, zz * psi).real)) <= 1e-12


def test_sweep_errors():
    be = B200SvBackend(seed=0, precision="f32")
    with pytest.raises(QubitOutOfRange):
        be.qaoa_sweep([(3, [(0, 3)])], [[0.1]], [[0.2]])
    with pytest.raises(DuplicateQubit):
        be.qaoa_sweep([(3, [(1, 1)])], [[0.1]], [[0.2]])
    with pytest.raises(NonFiniteParam):
        be.qaoa_sweep([(3, [(0, 1)])], [[float("nan")]], [[0.2]])
    with pytest.raises(TooManyQubits):
        be.qaoa_sweep([(27, [(0, 1)])], [[0.1]], [[0.2]])
