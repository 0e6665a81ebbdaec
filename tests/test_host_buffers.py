"""Host-memory plumbing of the fused entry points (no GPU needed): which
inputs count as host memory, how they are handed to the C ABI without a
copy, and which output buffers the host-buffer calls accept."""
import numpy as np
import torch

from cbmv_b200 import _dev


def test_host_inputs_are_recognised():
    assert _dev.is_host(np.zeros((4, 5), np.uint8))
    assert _dev.is_host(torch.zeros((4, 5), dtype=torch.uint8))
    assert not _dev.is_host([[0, 1]])


def test_host_arrays_are_passed_without_a_copy_when_they_can_be():
    t = torch.arange(20, dtype=torch.uint8).reshape(4, 5)
    assert _dev.host_array(t, np.uint8) is t
    a = np.arange(20, dtype=np.uint8).reshape(4, 5)
    assert _dev.host_array(a, np.uint8) is a
    assert _dev.host_ptr(a) == a.ctypes.data and _dev.host_ptr(t) == t.data_ptr()
    # other layouts and types become contiguous uint8 copies
    b = _dev.host_array(a.T, np.uint8)
    assert b.flags.c_contiguous and np.array_equal(b, a.T)
    c = _dev.host_array(t.to(torch.int32), np.uint8)
    assert c.dtype == torch.uint8 and torch.equal(c, t)


def test_host_output_buffers_are_checked():
    assert _dev.host_f32_buffer(np.empty((3, 4), np.float32), (3, 4))
    assert _dev.host_f32_buffer(torch.empty((3, 4)), (3, 4))
    assert not _dev.host_f32_buffer(np.empty((3, 4), np.float64), (3, 4))
    assert not _dev.host_f32_buffer(np.empty((4, 3), np.float32), (3, 4))
    assert not _dev.host_f32_buffer(np.empty((4, 3), np.float32).T, (3, 4))
    ro = np.empty((3, 4), np.float32)
    ro.flags.writeable = False
    assert not _dev.host_f32_buffer(ro, (3, 4))
    assert not _dev.host_f32_buffer(torch.empty((4, 3)).t(), (3, 4))
