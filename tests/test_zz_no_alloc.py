"""The allocation-free expectation entry point (``ps_expectation_device_noalloc``).

It serves callers that cannot allocate device memory themselves: they hand over the store's
packed keys and coefficients and an output slot in device memory they already own, and the
library reduces them with a fixed scratch array of its own.  Here the caller's buffers come
from torch; the result must match ``ps_expectation`` on a handle holding the same terms, on
two calls in a row (the second call reuses the scratch the first one left behind).
"""

import ctypes

import numpy as np
import pytest

import paulistrings_b200 as ps
from paulistrings_b200 import _lib, truncation, workloads

pytestmark = pytest.mark.gpu


def _device_store(num_qubits, dtype, seed):
    import torch

    g = ps.GpuPauliSum(num_qubits, dtype)
    x, z, c = workloads.random_observable(num_qubits, 4000, seed=seed)
    g.upload(x, z, c)
    g.propagate(workloads.random_pair_layers(num_qubits, 1, seed=seed), truncation.coeff(1e-9), "heisenberg")
    x, z, c = g.download()
    keys = np.ascontiguousarray(np.concatenate([x, z], axis=1)).view(np.int64)
    tkeys = torch.from_numpy(keys).cuda()
    tcoef = torch.from_numpy(c.astype(np.float64 if dtype == "f64" else np.float32)).cuda()
    return g, tkeys, tcoef


def _noalloc(tkeys, tcoef, dtype, width, state, num_qubits, out):
    import torch

    ax, az, neg = ps.product_basis(state, num_qubits, width)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    status = _lib.lib().ps_expectation_device_noalloc(
        tkeys.data_ptr(), tcoef.data_ptr(), _lib.PS_F64 if dtype == "f64" else _lib.PS_F32, width,
        tkeys.shape[0], ax.ctypes.data, az.ctypes.data, neg.ctypes.data, out.data_ptr(), stream)
    assert status == _lib.PS_OK
    torch.cuda.synchronize()
    return float(out.item())


@pytest.mark.parametrize("num_qubits,dtype", [(64, "f64"), (64, "f32"), (100, "f64"), (256, "f64"), (200, "f32")])
def test_noalloc_expectation_matches_the_handle_entry_point_twice(num_qubits, dtype):
    import torch

    g, tkeys, tcoef = _device_store(num_qubits, dtype, seed=3)
    W = ps.width_for(num_qubits)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    states = ["z+", "".join("01"[q % 2] for q in range(num_qubits))]
    for state in states:  # two calls in a row on the shared scratch
        want = g.expectation(state)
        got = _noalloc(tkeys, tcoef, dtype, W, state, num_qubits, out)
        assert got == pytest.approx(want, rel=1e-12, abs=1e-15), state
    # the first state again, after the scratch holds the second call's partials
    assert _noalloc(tkeys, tcoef, dtype, W, states[0], num_qubits, out) == pytest.approx(
        g.expectation(states[0]), rel=1e-12, abs=1e-15)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    one = np.zeros(1, np.uint64)
    status = _lib.lib().ps_expectation_device_noalloc(
        out.data_ptr(), out.data_ptr(), _lib.PS_F64, 1, _lib.NOALLOC_MAX_TERMS + 1,
        one.ctypes.data, one.ctypes.data, one.ctypes.data, out.data_ptr(), None)
    assert status == _lib.PS_ERR_INVALID


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_noalloc_rejects_misaligned_pointers_without_launching(dtype):
    """keys must be 16-byte aligned, coefficients aligned to their element size and the output to
    8 bytes: an offset view of a caller's buffer is refused with PS_ERR_INVALID before anything
    reaches the device, and a correct call right after still matches the handle's readout."""
    import torch

    g, tkeys, tcoef = _device_store(64, dtype, seed=5)
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    ax, az, neg = ps.product_basis("z+", 64, 1)
    fn = _lib.lib().ps_expectation_device_noalloc
    code = _lib.PS_F64 if dtype == "f64" else _lib.PS_F32
    n = tkeys.shape[0] - 1
    esize = tcoef.element_size()
    bad = [
        (tkeys.data_ptr() + 8, tcoef.data_ptr(), out.data_ptr()),          # keys off 16 bytes
        (tkeys.data_ptr(), tcoef.data_ptr() + esize // 2, out.data_ptr()),  # coefficients off their size
        (tkeys.data_ptr(), tcoef.data_ptr(), out.data_ptr() + 4),           # output off 8 bytes
    ]
    for keys, coef, o in bad:
        assert fn(keys, coef, code, 1, n, ax.ctypes.data, az.ctypes.data, neg.ctypes.data, o, None) == \
            _lib.PS_ERR_INVALID
    torch.cuda.synchronize()
    assert _noalloc(tkeys, tcoef, dtype, 1, "z+", 64, out[:1]) == pytest.approx(g.expectation("z+"), rel=1e-12,
                                                                                abs=1e-15)
