"""aleph_b200_sample_cumulative_noalloc (fixed device buffer, no allocation)
against the allocating aleph_b200_sample(CUMULATIVE), through the C ABI.

The bitstrings are integer results of the same kernels on the same state and
variates, so the tolerance is exact equality. Collected last (file name) and
independent of the other tests' state.
"""
import ctypes as ct

import numpy as np
import pytest

from aleph_b200 import abi, workloads
from aleph_b200.backend import B200SvBackend, run

pytestmark = pytest.mark.gpu


def fixed_sample(be, st, variates):
    v = np.ascontiguousarray(variates, dtype=np.float64)
    out = np.zeros(max(1, v.size), dtype=np.uint64)
    status = be.lib.aleph_b200_sample_cumulative_noalloc(
        be.handle, st.ptr, v.size, v.ctypes.data_as(ct.POINTER(ct.c_double)),
        out.ctypes.data_as(ct.POINTER(ct.c_uint64)))
    return status, out[: v.size]


def device_free_bytes():
    import torch

    free, _ = torch.cuda.mem_get_info(0)
    return free


@pytest.mark.parametrize("precision,n,shots", [("f64", 20, 4096), ("f32", 27, 2048)])
def test_fixed_buffer_sampling_matches_allocating_entry_point(precision, n, shots):
    be = B200SvBackend(seed=0, precision=precision)  # a fresh handle: the fixed buffer is reserved here
    st = run(be, workloads.brickwall(n, 3, seed=40 + n))
    u = np.random.default_rng(n).random(shots)
    want = be.sample(st, shots, variates=u, mode="cumulative")
    be.synchronize()
    free_before = device_free_bytes()
    for _ in range(2):  # two calls in a row reuse the same buffer
        status, got = fixed_sample(be, st, u)
        assert status == abi.OK
        assert np.array_equal(got, want)
    # nothing was allocated on the device by the two calls
    assert device_free_bytes() == free_before


def test_fixed_buffer_rejects_requests_over_its_size():
    be = B200SvBackend(seed=0, precision="f64")
    st = run(be, workloads.brickwall(12, 2, seed=3))
    status, _ = fixed_sample(be, st, np.full(1 << 20, 0.5))  # 8 MiB of variates alone
    assert status == abi.INVALID_ARGUMENT
    buf = ct.create_string_buffer(256)
    be.lib.aleph_b200_last_error(be.handle, buf, 256)
    assert b"fixed sampling buffer" in buf.value
    status, got = fixed_sample(be, st, np.array([0.25, 0.75]))  # still usable afterwards
    assert status == abi.OK
    assert np.array_equal(got, be.sample(st, 2, variates=[0.25, 0.75], mode="cumulative"))
