"""Device plumbing: PyTorch owns device memory and streams; kernels run through the C ABI."""

from __future__ import annotations

import threading

import numpy as np


def torch():
    import torch as _torch

    return _torch


def require_cuda():
    """Return the current CUDA device, raising if the B200 path cannot run."""

    t = torch()
    if not t.cuda.is_available():
        raise RuntimeError(
            "art_b200 requires a CUDA device (sm_100); no CPU fallback exists for this path."
        )
    return t.device("cuda", t.cuda.current_device())


def stream_handle(stream=None) -> int:
    t = torch()
    s = t.cuda.current_stream() if stream is None else stream
    return int(s.cuda_stream)


def ptr(tensor) -> int | None:
    if tensor is None:
        return None
    return int(tensor.data_ptr())


def to_device(array, dtype=None, device=None):
    """numpy / torch -> contiguous CUDA tensor (no copy if already suitable)."""

    t = torch()
    device = require_cuda() if device is None else device
    if isinstance(array, t.Tensor):
        out = array.to(device=device, dtype=dtype if dtype is not None else array.dtype)
        return out.contiguous()
    arr = np.ascontiguousarray(array, dtype=None if dtype is None else _np_dtype(dtype))
    if not arr.flags.writeable:  # read-only views (broadcasts, loaded buffers): torch wants a writable array
        arr = arr.copy()
    return t.from_numpy(arr).to(device=device, non_blocking=False).contiguous()


def _np_dtype(torch_dtype):
    t = torch()
    return {
        t.float64: np.float64,
        t.float32: np.float32,
        t.int64: np.int64,
        t.int32: np.int32,
        t.int8: np.int8,
        t.uint8: np.uint8,
    }[torch_dtype]


class _WorkspaceCache:
    """One growing byte buffer per (device, stream): workspaces must not be shared
    by calls that may overlap on the GPU."""

    def __init__(self):
        self._buffers = {}
        self._lock = threading.Lock()

    def get(self, nbytes: int, stream=None):
        t = torch()
        device = require_cuda()
        key = (device.index, stream_handle(stream))
        with self._lock:
            buf = self._buffers.get(key)
            if buf is None or buf.numel() < nbytes:
                size = max(int(nbytes), 1 << 16)
                if buf is not None:
                    size = max(size, 2 * buf.numel())
                buf = t.empty(size, dtype=t.uint8, device=device)
                self._buffers[key] = buf
            return buf


WORKSPACES = _WorkspaceCache()
