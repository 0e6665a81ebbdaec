"""Device-memory plumbing for the drop-in modules (torch is used only to
allocate device buffers and to name the current CUDA stream)."""
import numpy as np
import torch

_NP2T = {np.dtype(np.uint8): torch.uint8, np.dtype(np.float32): torch.float32,
         np.dtype(np.float64): torch.float64, np.dtype(np.int32): torch.int32,
         np.dtype(np.int64): torch.int64, np.dtype(np.uint32): torch.int32}


def require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("cbmv_b200 needs a CUDA device (B200, sm_100a); none is visible")


def stream_ptr():
    return torch.cuda.current_stream().cuda_stream


def ptr(t):
    return t.data_ptr() if t is not None else None


def is_device(a):
    return isinstance(a, torch.Tensor) and a.is_cuda


def to_device(a, dtype):
    """(device tensor of `dtype`, True if the input was host memory)."""
    require_cuda()
    if isinstance(a, torch.Tensor):
        t = a.to(device="cuda", dtype=_NP2T[np.dtype(dtype)])
        return t.contiguous(), not a.is_cuda
    arr = np.ascontiguousarray(a, dtype=dtype)
    t = torch.from_numpy(arr.view(np.int32) if arr.dtype == np.uint32 else arr)
    return t.to("cuda", non_blocking=False).contiguous(), True


def is_host(a):
    """True for numpy arrays and CPU tensors (pinned or not)."""
    return isinstance(a, np.ndarray) or (isinstance(a, torch.Tensor) and not a.is_cuda)


def host_array(a, dtype):
    """`a` as C-contiguous host memory of `dtype`: a numpy array, or a CPU
    tensor (kept as it is, pinned memory included, when it already is)."""
    if isinstance(a, torch.Tensor):
        return a.to(dtype=_NP2T[np.dtype(dtype)]).contiguous()
    return np.ascontiguousarray(a, dtype=dtype)


def host_f32_buffer(a, shape):
    """True when `a` can receive float32 [shape] results in place."""
    if isinstance(a, torch.Tensor):
        return a.dtype == torch.float32 and tuple(a.shape) == shape and a.is_contiguous()
    return a.dtype == np.float32 and a.shape == shape and a.flags.c_contiguous and a.flags.writeable


def host_ptr(a):
    return a.data_ptr() if isinstance(a, torch.Tensor) else a.ctypes.data


def empty(shape, dtype):
    require_cuda()
    return torch.empty(tuple(int(s) for s in shape), dtype=_NP2T[np.dtype(dtype)], device="cuda")


def zeros(shape, dtype):
    require_cuda()
    return torch.zeros(tuple(int(s) for s in shape), dtype=_NP2T[np.dtype(dtype)], device="cuda")


def result(t, host):
    """Returns `t` as numpy when the call's input came from the host."""
    if host:
        return t.cpu().numpy()
    return t
