"""Device-memory and stream plumbing (PyTorch tensors stand for device buffers)."""
from __future__ import annotations

import numpy as np
import torch


def require_cuda() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("the transport path runs on a CUDA GPU only (no CPU fallback)")
    return torch.device("cuda", torch.cuda.current_device())


def stream_handle(stream: torch.cuda.Stream | None = None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def ptr(t: torch.Tensor | None):
    return None if t is None else t.data_ptr()


def to_device(a, dtype: torch.dtype, device) -> torch.Tensor:
    """Contiguous device tensor of `dtype` from numpy / torch / list input (H2D if needed)."""
    if isinstance(a, torch.Tensor):
        return a.to(device=device, dtype=dtype).contiguous()
    if hasattr(a, "__cuda_array_interface__"):
        return torch.as_tensor(a, device=device).to(dtype).contiguous()
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a), dtype=_np_dtype(dtype))).to(device)


def _np_dtype(dtype: torch.dtype):
    return {torch.float64: np.float64, torch.float32: np.float32, torch.int32: np.int32,
            torch.int64: np.int64, torch.uint8: np.uint8}[dtype]


def empty_aligned(nbytes: int, device, align: int = 256) -> tuple[torch.Tensor, int]:
    """Byte buffer plus an address inside it aligned to `align`."""
    buf = torch.empty(int(nbytes) + align, dtype=torch.uint8, device=device)
    base = buf.data_ptr()
    off = (-base) % align
    return buf, base + off


def length(a) -> int:
    return int(a.shape[0])
