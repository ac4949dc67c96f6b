"""Amplitude sharding through the engine on one GPU: 2^g virtual ranks as
engine states on cuda:0, local steps run by the engine's gate streams and
exchanges as device copies between the ranks' halves (the in-process path
of aleph_b200/dist.py's Exchange), against the oracle. Runs of one rank per
GPU over NCCL are unmeasured here: every run has one GPU (their
torch.distributed path is tested over gloo in tests/test_cpu_dist.py)."""
import numpy as np
import pytest

from aleph_b200 import circuit as C
from aleph_b200 import dist, workloads
from aleph_b200.backend import B200SvBackend
from oracle import oracle
from tests.circuit_gen import random_circuit
from tests.test_cpu_dist import phase_circuit

pytestmark = pytest.mark.gpu


def sharded(circ, g, precision="f64", chunk=1 << 20):
    be = B200SvBackend(seed=0, precision=precision)
    st = dist.run_distributed(circ, g, be, chunk_bytes=chunk)
    got = dist.gather_statevector(st)
    norm = dist.norm_sqr(st)
    ex = st.stats["exchanges"]
    st.ranks.free()
    be.close()
    return got, norm, ex


@pytest.mark.parametrize("g", [1, 2, 3])
@pytest.mark.parametrize("name,make", [
    ("random", lambda: random_circuit(14, 260, seed=91)),
    ("qft", lambda: workloads.qft_product(14, seed=92)),
    ("brickwall", lambda: workloads.brickwall(14, 12, seed=93)),
    ("phase", lambda: phase_circuit(14, 94)),
])
def test_sharded_engine_run_matches_oracle(name, make, g):
    c = make()
    want, _ = oracle.run(14, c.instructions)
    got, norm, ex = sharded(c, g)
    assert np.abs(got - want).max() <= 1e-12
    assert abs(norm - 1.0) <= 1e-12
    if name != "phase":
        assert ex > 0


@pytest.mark.parametrize("precision", ["f32", "tc32"])
def test_sharded_single_precision(precision):
    c = workloads.brickwall(16, 10, seed=95)
    want, _ = oracle.run(16, c.instructions)
    got, norm, _ = sharded(c, 2, precision)
    assert np.abs(got - want).max() <= 1e-5
    assert abs(norm - 1.0) <= 1e-5


def test_sharded_large_slices_chunked_exchange():
    # 4 ranks of 2^22 amplitudes (64 MiB each), exchanged in 4 MiB chunks
    n = 24
    c = workloads.brickwall(n, 8, seed=96)
    want, _ = oracle.run(n, c.instructions)
    got, norm, ex = sharded(c, 2, chunk=4 << 20)
    assert ex > 0
    assert np.abs(got - want).max() <= 1e-12


def test_handle_renormalises_again_after_a_sharded_tc32_run():
    be = B200SvBackend(seed=0, precision="tc32")
    st = dist.run_distributed(workloads.brickwall(14, 6, seed=97), 1, be)
    st.ranks.free()
    c = workloads.brickwall(16, 20, seed=98)
    s = be.allocate(16)
    be.apply_stream(s, c.instructions)
    # the end-of-stream rescale ran: FP32 rounding only (a TC32 stream without
    # it drifts by about 1e-6 per block pass)
    assert abs(be.norm_sqr(s) - 1.0) <= 1e-6
    s.free()
    be.close()
