"""Thin CUDA-runtime plumbing (device buffers, streams, events, pinned host
memory) over cuda-python, for callers that drive the ``*_async`` device-
pointer entry points.  No kernels here: the march itself is the C library.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
from cuda.bindings import runtime as rt


def _ok(res):
    err = res[0] if isinstance(res, tuple) else res
    if err != rt.cudaError_t.cudaSuccess:
        raise RuntimeError(f"CUDA runtime error: {err}")
    if isinstance(res, tuple):
        return res[1] if len(res) == 2 else res[1:]
    return None


def set_device(i: int) -> None:
    _ok(rt.cudaSetDevice(i))


def synchronize() -> None:
    _ok(rt.cudaDeviceSynchronize())


class DeviceArray:
    """A device allocation with a numpy dtype and element count."""

    def __init__(self, n: int, dtype):
        self.dtype = np.dtype(dtype)
        self.n = int(n)
        self.nbytes = max(1, self.n * self.dtype.itemsize)
        self.ptr = int(_ok(rt.cudaMalloc(self.nbytes)))

    def upload(self, host: np.ndarray, stream=None):
        host = np.ascontiguousarray(host, self.dtype)
        assert host.nbytes <= self.nbytes
        if stream is None:
            _ok(rt.cudaMemcpy(self.ptr, host.ctypes.data, host.nbytes, rt.cudaMemcpyKind.cudaMemcpyHostToDevice))
        else:
            _ok(rt.cudaMemcpyAsync(self.ptr, host.ctypes.data, host.nbytes,
                                   rt.cudaMemcpyKind.cudaMemcpyHostToDevice, stream.handle))
        return self

    def download(self) -> np.ndarray:
        out = np.empty(self.n, self.dtype)
        _ok(rt.cudaMemcpy(out.ctypes.data, self.ptr, out.nbytes, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost))
        return out

    def download_into(self, host: np.ndarray, stream=None) -> np.ndarray:
        """Copy the first host.size elements into ``host`` (asynchronously on
        ``stream`` when given: ``host`` should then be page-locked)."""
        assert host.dtype == self.dtype and host.flags.c_contiguous and host.nbytes <= self.nbytes
        if stream is None:
            _ok(rt.cudaMemcpy(host.ctypes.data, self.ptr, host.nbytes, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost))
        else:
            _ok(rt.cudaMemcpyAsync(host.ctypes.data, self.ptr, host.nbytes,
                                   rt.cudaMemcpyKind.cudaMemcpyDeviceToHost, stream.handle))
        return host

    def memset(self, value: int = 0, stream=None):
        if stream is None:
            _ok(rt.cudaMemset(self.ptr, value, self.nbytes))
        else:
            _ok(rt.cudaMemsetAsync(self.ptr, value, self.nbytes, stream.handle))

    def free(self):
        if self.ptr:
            rt.cudaFree(self.ptr)
            self.ptr = 0

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class PinnedArray:
    """Page-locked host memory viewed as a numpy array."""

    def __init__(self, n: int, dtype):
        self.dtype = np.dtype(dtype)
        nbytes = max(1, int(n) * self.dtype.itemsize)
        self.ptr = int(_ok(rt.cudaMallocHost(nbytes)))
        buf = (C.c_char * nbytes).from_address(self.ptr)
        self.array = np.frombuffer(buf, dtype=self.dtype, count=int(n))

    def free(self):
        if self.ptr:
            rt.cudaFreeHost(self.ptr)
            self.ptr = 0

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Stream:
    def __init__(self):
        self.handle = _ok(rt.cudaStreamCreateWithFlags(rt.cudaStreamNonBlocking))

    @property
    def ptr(self) -> int:
        return int(self.handle)

    def synchronize(self):
        _ok(rt.cudaStreamSynchronize(self.handle))


class Event:
    def __init__(self):
        self.handle = _ok(rt.cudaEventCreate())

    def record(self, stream: Stream):
        _ok(rt.cudaEventRecord(self.handle, stream.handle))

    def elapsed_ms(self, end: "Event") -> float:
        return float(_ok(rt.cudaEventElapsedTime(self.handle, end.handle)))


def device_gbuffer(n: int, reference_planes: bool = False) -> dict:
    g = {"t": DeviceArray(n, np.float32), "normal": DeviceArray(3 * n, np.float32),
         "slot": DeviceArray(n, np.uint32), "material": DeviceArray(n, np.uint16),
         "flags": DeviceArray(n, np.uint16)}
    if reference_planes:
        g["position"] = DeviceArray(4 * n, np.float32)
        g["packed_material"] = DeviceArray(n, np.uint32)
        g["motion"] = DeviceArray(4 * n, np.float32)
    return g


def gbuffer_ptrs(g: dict) -> dict:
    return {k: v.ptr for k, v in g.items()}
