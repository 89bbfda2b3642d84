"""FP64 vector primitives on flat device buffers (through the C ABI)."""

from __future__ import annotations

import torch

from tenax_b200 import _capi

_SCRATCH: dict = {}


def _stream_ptr() -> int:
    return torch.cuda.current_stream().cuda_stream


def scratch(device=None) -> torch.Tensor:
    """Per-device reduction scratch (tnx_reduce_scratch_len doubles)."""
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else device
    key = (dev.index, _stream_ptr())
    buf = _SCRATCH.get(key)
    if buf is None:
        buf = torch.empty(int(_capi.LIB.tnx_reduce_scratch_len()), dtype=torch.float64, device=dev)
        _SCRATCH[key] = buf
    return buf


def dot(x: torch.Tensor, y: torch.Tensor) -> torch.Tensor:
    out = torch.empty((), dtype=torch.float64, device=x.device)
    _capi.check(_capi.LIB.tnx_dot(x.data_ptr(), y.data_ptr(), x.numel(), out.data_ptr(),
                                  scratch(x.device).data_ptr(), _stream_ptr()))
    return out


def nrm2(x: torch.Tensor) -> torch.Tensor:
    out = torch.empty((), dtype=torch.float64, device=x.device)
    _capi.check(_capi.LIB.tnx_nrm2(x.data_ptr(), x.numel(), out.data_ptr(), scratch(x.device).data_ptr(),
                                   _stream_ptr()))
    return out


def scale(x: torch.Tensor, s: torch.Tensor, mode: int, out: torch.Tensor | None = None) -> torch.Tensor:
    """mode 0: x*s, 1: x/s, 2: x*(1/(s+1e-15)); s is a device scalar."""
    if out is None:
        out = torch.empty_like(x)
    _capi.check(_capi.LIB.tnx_scale(x.data_ptr(), out.data_ptr(), x.numel(), s.data_ptr(), mode, _stream_ptr()))
    return out
