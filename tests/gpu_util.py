"""Device-buffer helpers for the GPU tests (torch is only the allocator)."""
import ctypes

import numpy as np
import torch

import arbor_b200 as ab


def dev(a: np.ndarray) -> torch.Tensor:
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint32:
        t = torch.from_numpy(a.view(np.int32).copy())
    else:
        t = torch.from_numpy(a.copy())
    return t.cuda()


def host(t: torch.Tensor, dtype=None) -> np.ndarray:
    torch.cuda.synchronize()
    a = t.cpu().numpy()
    if dtype is not None:
        a = a.view(dtype)
    return a


def zeros_f(n: int) -> torch.Tensor:
    return torch.zeros(n, dtype=torch.float32, device="cuda")


def zeros_u(n: int) -> torch.Tensor:
    return torch.zeros(n, dtype=torch.int32, device="cuda")


def ok(status: int) -> None:
    assert status == ab.OK, f"{ab.STATUS.get(status)}: {ab.last_error()}"


class DevScene:
    """A scene's ABI buffers on the device."""

    def __init__(self, scene: dict | None = None):
        self.B = zeros_f(2109 * 20)
        self.P = zeros_f(32768 * 24)
        self.Keys = zeros_u(32768)
        self.Order = zeros_u(32768)
        self.Nodes = zeros_f(65536 * 8)
        if scene is not None:
            for k in ("B", "P", "Keys", "Order", "Nodes"):
                getattr(self, k).copy_(dev(scene[k]))


def render_buffers(w: int, h: int) -> dict:
    return {k: zeros_f(w * h * 4) for k in ("Hit", "Linear", "Guide", "Filtered", "History")} | {"Pixels": zeros_u(w * h)}


def ulp_diff(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Distance in float32 units-in-the-last-place (same-sign values)."""
    ai = np.ascontiguousarray(a, np.float32).view(np.int32).astype(np.int64)
    bi = np.ascontiguousarray(b, np.float32).view(np.int32).astype(np.int64)
    ai = np.where(ai < 0, -(ai & 0x7FFFFFFF), ai)
    bi = np.where(bi < 0, -(bi & 0x7FFFFFFF), bi)
    return np.abs(ai - bi)


def rel_err(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """|a - b| / max(1, |b|): absolute error below magnitude 1, relative above."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) / np.maximum(1.0, np.abs(b))


_RT = None


def _cudart():
    """The CUDA runtime torch itself loaded (used only to copy library-owned buffers out)."""
    global _RT
    if _RT is None:
        import glob
        import os

        base = os.path.join(os.path.dirname(torch.__file__), "..", "nvidia")
        cands = sorted(glob.glob(os.path.join(base, "cuda_runtime", "lib", "libcudart.so*")))
        cands += ["libcudart.so.12", "/usr/local/cuda/lib64/libcudart.so"]
        for c in cands:
            try:
                _RT = ctypes.CDLL(c)
                break
            except OSError:
                continue
        _RT.cudaMemcpy.restype = ctypes.c_int
        _RT.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    return _RT


def dev_array(ptr: int, n: int, dtype=np.float32) -> np.ndarray:
    """Copy n 4-byte elements at a library-owned device address to the host."""
    torch.cuda.synchronize()
    out = np.empty(n, dtype)
    assert _cudart().cudaMemcpy(out.ctypes.data, ptr, n * 4, 2) == 0  # cudaMemcpyDeviceToHost
    return out


def dev_bits(ptr: int, n: int) -> torch.Tensor:
    """Copy n 4-byte elements at a library-owned device address into a new
    int32 device tensor (the bit patterns, for exact comparison on the GPU)."""
    torch.cuda.synchronize()
    out = torch.empty(n, dtype=torch.int32, device="cuda")
    assert _cudart().cudaMemcpy(out.data_ptr(), ptr, n * 4, 3) == 0  # cudaMemcpyDeviceToDevice
    return out
