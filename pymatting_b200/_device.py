"""Device-buffer plumbing: torch tensors hold device memory, the CUDA library
computes. Nothing here does arithmetic on the data."""

import numpy as np
import torch

_DTYPES = {np.dtype(np.float64): torch.float64, np.dtype(np.float32): torch.float32,
           np.dtype(np.uint8): torch.uint8, np.dtype(np.int64): torch.int64,
           np.dtype(np.bool_): torch.bool}


class NoDeviceError(RuntimeError):
    """pymatting_b200 computes only on a CUDA device and found none."""


def device():
    if not torch.cuda.is_available():
        raise NoDeviceError(
            "pymatting_b200 needs a CUDA device (B200, sm_100a); it has no CPU fallback")
    return torch.device("cuda", torch.cuda.current_device())


def stream():
    """Handle of the current torch stream, passed to the library as void*."""
    return torch.cuda.current_stream().cuda_stream


def ptr(t):
    return None if t is None else t.data_ptr()


def empty(shape, dtype):
    return torch.empty(shape, dtype=dtype, device=device())


def zeros(shape, dtype):
    return torch.zeros(shape, dtype=dtype, device=device())


def is_device_tensor(a):
    return isinstance(a, torch.Tensor) and a.is_cuda


def to_device(a, dtype=None):
    """Host array or device tensor -> contiguous device tensor of `dtype`."""
    if isinstance(a, torch.Tensor):
        t = a
        if dtype is not None and t.dtype != dtype:
            t = t.to(dtype)
        if not t.is_cuda:
            t = t.to(device())
        return t.contiguous()
    arr = np.ascontiguousarray(a)
    if arr.dtype == np.bool_:
        arr = arr.view(np.uint8)
    t = torch.from_numpy(arr)
    if dtype is not None and t.dtype != dtype:
        t = t.to(dtype)
    return t.to(device(), non_blocking=False).contiguous()


def to_host(t):
    torch.cuda.current_stream().synchronize()
    return t.detach().cpu().numpy()


def workspace(nbytes):
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=device())
