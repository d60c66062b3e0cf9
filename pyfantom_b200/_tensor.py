"""Array conversion helpers: everything the library touches is a contiguous CUDA tensor."""
from __future__ import annotations

import numpy as np
import torch


def device() -> torch.device:
    return torch.device("cuda", torch.cuda.current_device())


def to_torch_dtype(dtype) -> torch.dtype:
    if isinstance(dtype, torch.dtype):
        return dtype
    return {np.dtype(np.float64): torch.float64, np.dtype(np.float32): torch.float32,
            np.dtype(np.int32): torch.int32, np.dtype(np.int64): torch.int64,
            np.dtype(np.bool_): torch.bool}[np.dtype(dtype)]


def as_cuda(x, dtype=None) -> torch.Tensor:
    """Contiguous CUDA tensor view/copy of a tensor, numpy array, DLPack object or scalar list."""
    td = to_torch_dtype(dtype) if dtype is not None else None
    if isinstance(x, torch.Tensor):
        t = x
    elif isinstance(x, np.ndarray):
        t = torch.from_numpy(np.ascontiguousarray(x))
    elif hasattr(x, "__dlpack__"):
        t = torch.from_dlpack(x)
    else:
        t = torch.as_tensor(np.asarray(x))
    if td is not None and t.dtype != td:
        t = t.to(td)
    if not t.is_cuda:
        t = t.to(device(), non_blocking=False)
    return t.contiguous()


def is_cuda_vector(x) -> bool:
    return isinstance(x, torch.Tensor) and x.is_cuda
