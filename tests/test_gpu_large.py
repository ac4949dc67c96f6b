"""Parity at the sizes of the benchmark configurations, through the C ABI.

* The depth-40 random brickwall at n=28 (the oracle copy of the n=32
  headline circuit) against the raw FP64 oracle: the plain FP64 path to
  max|dpsi| <= 1e-12, the tensor-core FP32 path (split-BF16x3 blocks) to
  1 - fidelity <= 1e-6. The oracle needs 4 GiB of host memory and a few
  minutes on the host cores.
* In-core states at the top of the engine's range, n=33 FP64 and n=34 FP32
  (128 GiB each, above the reference's caps of 30 / 31,
  crates/aleph-backend/src/select.rs:36,40), on a circuit whose amplitudes
  have a closed form: Ry(theta_q) Rz(phi_q) on every qubit, then CZ on every
  nearest-neighbour pair, so
      psi(x) = prod_q a_q(x_q) * (-1)^(sum_i x_i x_{i+1}).
  Amplitude windows (below and above 2^32), the FP64 norm, marginals of
  qubits up to n-1, and 1024 CUMULATIVE shots (each sampled index x must
  satisfy CDF(x-1) <= u <= CDF(x), the CDF of the product distribution in
  closed form) are checked.
"""
import numpy as np
import pytest

from aleph_b200 import circuit as C
from aleph_b200 import workloads
from aleph_b200.backend import B200SvBackend
from oracle import oracle

pytestmark = pytest.mark.gpu


def fidelity(a, b):
    return abs(np.vdot(a, b)) ** 2 / (np.vdot(a, a).real * np.vdot(b, b).real)


def test_brickwall_n28_depth40_against_the_oracle():
    n, depth = 28, 40
    c = workloads.brickwall(n, depth, seed=0)
    want, _ = oracle.run(n, c.instructions)
    be = B200SvBackend(seed=0, precision="f64")
    st = be.allocate(n)
    be.apply_stream(st, c.instructions)
    got = be.statevector(st)
    st.free()
    be.close()
    assert np.abs(got - want).max() <= 1e-12
    del got
    tc = B200SvBackend(seed=0, precision="tc32")
    st = tc.allocate(n)
    tc.apply_stream(st, c.instructions)
    assert tc.stats()["block_passes"] > 0
    got = tc.statevector(st)
    st.free()
    tc.close()
    assert 1.0 - fidelity(want, got) <= 1e-6
    assert np.abs(got - want).max() <= 1e-5


def product_circuit(n, seed):
    rng = np.random.default_rng(seed)
    theta = rng.uniform(0.3, 2.8, n)
    phi = rng.uniform(-3.0, 3.0, n)
    c = C.Circuit(n)
    for q in range(n):
        c.add(C.Ry(theta[q]), [q]).add(C.Rz(phi[q]), [q])
    for off in (0, 1):
        for q in range(off, n - 1, 2):
            c.add(C.Cz(), [q, q + 1])
    # per-qubit amplitudes from the gate matrices the engine implements
    a = np.zeros((n, 2), dtype=np.complex128)
    for q in range(n):
        ry = oracle.gate_matrix(C.GateInstance(C.Ry(theta[q]), [0]))
        rz = oracle.gate_matrix(C.GateInstance(C.Rz(phi[q]), [0]))
        a[q] = rz @ ry @ np.array([1.0, 0.0])
    return c, a


def closed_form(a, idx):
    n = a.shape[0]
    idx = np.asarray(idx, dtype=np.uint64)
    bits = ((idx[:, None] >> np.arange(n, dtype=np.uint64)[None, :]) & np.uint64(1)).astype(np.int64)
    amp = np.prod(a[np.arange(n)[None, :], bits], axis=1)
    par = np.sum(bits[:, :-1] * bits[:, 1:], axis=1) & 1
    return amp * np.where(par == 1, -1.0, 1.0)


def cdf(p, x):
    """P(Y <= x) for independent bits with P(bit_q = 1) = p[q], index bit q = qubit q."""
    n = p.size
    below, above = 0.0, 1.0  # `above`: probability that bits above q equal x's
    for q in range(n - 1, -1, -1):
        b = (x >> q) & 1
        if b:
            below += above * (1.0 - p[q])
        above *= p[q] if b else 1.0 - p[q]
    return below + above


@pytest.mark.parametrize("precision,n", [("f64", 33), ("f32", 34), ("tc32", 34)])
def test_in_core_top_of_range(precision, n):
    c, a = product_circuit(n, seed=n)
    be = B200SvBackend(seed=0, precision=precision)
    st = be.allocate(n)
    be.apply_stream(st, c.instructions)
    tol_rel = 1e-12 if precision == "f64" else 1e-5
    scale = float(np.prod(np.abs(a).max(axis=1)))  # the largest amplitude
    rng = np.random.default_rng(1)
    starts = [0, (1 << 32) - 2048, 1 << 32, (1 << 32) + 777777, (1 << n) - 4096,
              int(rng.integers(0, (1 << n) - 4096))]
    for first in starts:
        got = be.amplitude_range(st, first, 4096)
        want = closed_form(a, np.arange(first, first + 4096, dtype=np.uint64))
        assert np.abs(got - want).max() <= tol_rel * scale, first
    assert abs(be.norm_sqr(st) - 1.0) <= (1e-10 if precision == "f64" else 1e-5)
    p1 = np.abs(a[:, 1]) ** 2
    qs = sorted({0, 17, 31, 32, n - 1})
    marg = be.probabilities(st, qs)
    for j in range(1 << len(qs)):
        want = np.prod([p1[q] if (j >> k) & 1 else 1.0 - p1[q] for k, q in enumerate(qs)])
        assert abs(marg[j] - want) <= (1e-12 if precision == "f64" else 1e-5)
    u = np.random.default_rng(2).random(1024)
    s0 = be.stats()
    shots = be.sample(st, 1024, variates=u, mode="cumulative")
    s1 = be.stats()
    tol = 1e-9 if precision == "f64" else 1e-5
    for x, ui in zip(shots.tolist(), u):
        assert x < (1 << n)
        lo = cdf(p1, x - 1) if x > 0 else 0.0
        assert lo - tol <= ui <= cdf(p1, x) + tol
    # above n = 28 every guard-band shot is reported as not re-resolved exactly
    gb = s1["guard_band_shots"] - s0["guard_band_shots"]
    assert s1["guard_band_inexact"] - s0["guard_band_inexact"] == gb
    st.free()
    be.close()
