"""ctypes binding of libfvx.so, the package's C-ABI CUDA library.

Every public operator in this package calls one of the ``fvx_*`` entry
points declared in ``include/fvx.h``.  There is no CPU or pure-torch
fallback: if the library is missing, or no CUDA device is present, calls
fail with a RuntimeError.
"""

from __future__ import annotations

import ctypes
import os
import pathlib

import numpy as np
import torch

_HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = _HERE / "libfvx.so"

FVX_OK = 0
_STATUS_TEXT = {
    1: "shape or size out of the supported range",
    2: "unknown method / operator",
    3: "unsupported dtype",
    4: "CUDA error",
    5: "solver did not converge",
    6: "invalid argument",
    7: "device-side wait timed out",
}

SCHEMES = {
    "naive": 0, "upwind1": 1, "upwind2": 2, "upwind3": 3, "weno3": 4, "weno5": 5, "wenoz5": 6,
    "weno7": 7, "weno9": 8, "minmod": 9, "van_leer": 10, "superbee": 11, "mc": 12, "wenoz3": 13,
}

_lib = None


class FvxError(RuntimeError):
    pass


def lib() -> ctypes.CDLL:
    """Load libfvx.so once; raise loudly if it is absent."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m finitevolx_b200.build` "
                "(finitevolx_b200 has no CPU fallback)")
        _lib = ctypes.CDLL(str(LIB_PATH))
    return _lib


def check(status: int, what: str) -> None:
    if status != FVX_OK:
        detail = _STATUS_TEXT.get(status, f"status {status}")
        if status == 4:
            err = torch.cuda.current_device() if torch.cuda.is_available() else "n/a"
            detail += f" (device {err})"
        raise FvxError(f"{what}: {detail}")


def require_cuda() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("finitevolx_b200 needs a CUDA device (B200, sm_100a); none is visible")
    return torch.device("cuda", torch.cuda.current_device())


def stream_ptr() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def P(t) -> ctypes.c_void_p:
    """Device pointer of a tensor (None -> NULL)."""
    if t is None:
        return ctypes.c_void_p(0)
    return ctypes.c_void_p(t.data_ptr())


def as_field(x, dtype=None, device=None) -> torch.Tensor:
    """Bring an array-like onto the CUDA device as a contiguous tensor."""
    dev = device or require_cuda()
    if isinstance(x, torch.Tensor):
        t = x
        if dtype is not None and t.dtype != dtype:
            t = t.to(dtype)
        if t.device != dev:
            t = t.to(dev)
        return t.contiguous()
    arr = np.asarray(x)
    if dtype is None:
        dtype = torch.float64 if arr.dtype == np.float64 else (
            torch.float32 if arr.dtype == np.float32 else None)
    t = torch.as_tensor(arr)
    if dtype is not None:
        t = t.to(dtype)
    return t.to(dev).contiguous()


def as_mask(m, device=None):
    """bool/0-1 mask -> contiguous uint8 (torch.bool) device tensor, or None."""
    if m is None:
        return None
    dev = device or require_cuda()
    if isinstance(m, torch.Tensor):
        t = m.to(dev)
        if t.dtype != torch.bool:
            t = t != 0
        return t.contiguous()
    return torch.as_tensor(np.asarray(m) != 0).to(dev).contiguous()


def sfx(t: torch.Tensor) -> str:
    if t.dtype == torch.float32:
        return "f32"
    if t.dtype == torch.float64:
        return "f64"
    raise TypeError(f"unsupported dtype {t.dtype}; finitevolx_b200 computes in float32 or float64")


def fn(name: str):
    return getattr(lib(), name)


D = ctypes.c_double
I = ctypes.c_int
I64 = ctypes.c_int64
