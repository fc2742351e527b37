"""Learned warm start: the message-passing network that predicts LOBPCG's
starting block (no counterpart in the spectral-init crate, whose LOBPCG starts
from a seeded random block, ``src/solvers/lobpcg.rs:244-291``).

The network's forward pass, backward pass and Adam update run in
``libspectral_init_b200.so`` (``mpnn.cu``: bf16 tcgen05 GEMMs for the dense
layers, warp-per-row CSR message passing).  This module holds the Python side:
a device-resident Laplacian to train or predict on, the model handle, and the
weights file format (``SIWS`` magic, version, parameter count, little-endian
f32 parameters).
"""
from __future__ import annotations

import ctypes as C
import struct
from pathlib import Path

import numpy as np

from . import _lib
from ._lib import SiCsrF32, SiOperator
from .api import Context, as_csr_f32, get_context, _torch

WEIGHTS_PATH = Path(__file__).resolve().parent / "warm_start_weights.bin"
_MAGIC = b"SIWS"
_VERSION = 1


class DeviceLaplacian:
    """Graph, degrees and the implicit-unit-diagonal Laplacian held on the device.

    ``graph`` is anything ``as_csr_f32`` accepts, or a tuple of torch CUDA
    tensors ``(indptr int64, indices int32, data float32, n)`` already on the
    device.  ``op()`` is the ``si_operator`` (diag 1, f64 and f32 values).
    """

    def __init__(self, graph, *, ctx: Context | None = None, mode: int = 0):
        self.ctx = ctx or get_context()
        torch = _torch()
        dev = torch.device("cuda", self.ctx.device)
        if isinstance(graph, tuple) and len(graph) == 4 and hasattr(graph[0], "data_ptr"):
            self.indptr, self.indices, self.data, self.n = graph
        else:
            n, ip, ix, dv = as_csr_f32(graph)
            self.n = n
            self.indptr = torch.from_numpy(ip.view(np.int64)).to(dev)
            self.indices = torch.from_numpy(ix.view(np.int32)).to(dev)
            self.data = torch.from_numpy(dv).to(dev)
        self.nnz = int(self.indices.numel())
        g = SiCsrF32(self.n, self.nnz, self.indptr.data_ptr(), self.indices.data_ptr(), self.data.data_ptr())
        self.deg = torch.empty(self.n, dtype=torch.float64, device=dev)
        self.sqrt_deg = torch.empty_like(self.deg)
        torch.cuda.synchronize(dev)
        lib = self.ctx.lib
        self.ctx.check(lib.si_compute_degrees(self.ctx.ptr, C.byref(g), int(mode), self.deg.data_ptr(),
                                              self.sqrt_deg.data_ptr()))
        inv = torch.where(self.sqrt_deg > 0, 1.0 / self.sqrt_deg, torch.zeros_like(self.sqrt_deg))
        self.v64 = torch.empty(max(self.nnz, 1), dtype=torch.float64, device=dev)
        self.v32 = torch.empty(max(self.nnz, 1), dtype=torch.float32, device=dev)
        torch.cuda.synchronize(dev)
        self.ctx.check(lib.si_build_laplacian(self.ctx.ptr, C.byref(g), inv.data_ptr(), self.v64.data_ptr(),
                                              self.v32.data_ptr()))

    def op(self) -> SiOperator:
        return SiOperator(self.n, self.nnz, self.indptr.data_ptr(), self.indices.data_ptr(), self.v64.data_ptr(),
                          self.v32.data_ptr(), 1.0)


def param_count() -> int:
    return int(_lib.load().si_model_param_count())


def save_params(path, params: np.ndarray) -> None:
    p = np.ascontiguousarray(params, dtype="<f4")
    with open(path, "wb") as f:
        f.write(_MAGIC + struct.pack("<II", _VERSION, p.size))
        f.write(p.tobytes())


def load_params(path) -> np.ndarray:
    raw = Path(path).read_bytes()
    if raw[:4] != _MAGIC:
        raise ValueError(f"{path}: not a warm-start weights file")
    version, count = struct.unpack("<II", raw[4:12])
    if version != _VERSION or count != param_count():
        raise ValueError(f"{path}: version {version} with {count} parameters, expected {_VERSION}/{param_count()}")
    return np.frombuffer(raw[12:12 + 4 * count], dtype="<f4").astype(np.float32)


class WarmStartModel:
    """Handle of one network on the context's device (``si_model``)."""

    def __init__(self, seed: int = 0, *, ctx: Context | None = None, params: np.ndarray | None = None):
        self.ctx = ctx or get_context()
        self.lib = self.ctx.lib
        self.ptr = C.c_void_p()
        self.ctx.check(self.lib.si_model_create(self.ctx.ptr, int(seed), C.byref(self.ptr)))
        if params is not None:
            self.set_params(params)

    @classmethod
    def load(cls, path=None, *, ctx: Context | None = None) -> "WarmStartModel":
        return cls(ctx=ctx, params=load_params(path or WEIGHTS_PATH))

    def save(self, path) -> None:
        save_params(path, self.get_params())

    def get_params(self) -> np.ndarray:
        out = np.empty(param_count(), dtype=np.float32)
        self.ctx.check(self.lib.si_model_get_params(self.ctx.ptr, self.ptr, out.ctypes.data_as(C.c_void_p)))
        return out

    def set_params(self, params: np.ndarray) -> None:
        p = np.ascontiguousarray(params, dtype=np.float32)
        if p.size != param_count():
            raise ValueError(f"expected {param_count()} parameters, got {p.size}")
        self.ctx.check(self.lib.si_model_set_params(self.ctx.ptr, self.ptr, p.ctypes.data_as(C.c_void_p)))

    def train_step(self, lap: DeviceLaplacian, target, seed: int, lr: float) -> float:
        """One Adam step; ``target`` is a torch f64 CUDA tensor [n, k] (orthonormal)."""
        target = target.contiguous()
        loss = C.c_double(0.0)
        _torch().cuda.synchronize()
        self.ctx.check(self.lib.si_model_train_step(self.ctx.ptr, self.ptr, C.byref(lap.op()),
                                                    lap.sqrt_deg.data_ptr(), target.data_ptr(), target.shape[1],
                                                    int(seed), float(lr), C.byref(loss)))
        return loss.value

    def gradient(self, lap: DeviceLaplacian, target, *, features=None, seed: int = 0):
        """(loss, flat gradient) without an update; ``features`` f32 CUDA [n, 5] or None."""
        target = target.contiguous()
        grad = np.empty(param_count(), dtype=np.float32)
        loss = C.c_double(0.0)
        _torch().cuda.synchronize()
        self.ctx.check(self.lib.si_model_gradient(
            self.ctx.ptr, self.ptr, C.byref(lap.op()), lap.sqrt_deg.data_ptr(),
            features.contiguous().data_ptr() if features is not None else None, target.data_ptr(),
            target.shape[1], int(seed), C.byref(loss), grad.ctypes.data_as(C.c_void_p)))
        return loss.value, grad

    def predict(self, lap: DeviceLaplacian, *, features=None, seed: int = 0):
        """Prediction Y (torch f32 CUDA [n, 16])."""
        torch = _torch()
        out = torch.empty(lap.n, 16, dtype=torch.float32, device=f"cuda:{self.ctx.device}")
        torch.cuda.synchronize()
        self.ctx.check(self.lib.si_model_predict(self.ctx.ptr, self.ptr, C.byref(lap.op()), lap.sqrt_deg.data_ptr(),
                                                 features.contiguous().data_ptr() if features is not None else None,
                                                 int(seed), out.data_ptr()))
        return out

    def attach(self) -> None:
        """Use this network for solves with ``warm_start=WarmStart.Learned`` on its context."""
        self.ctx.check(self.lib.si_ctx_set_model(self.ctx.ptr, self.ptr))

    def detach(self) -> None:
        self.ctx.check(self.lib.si_ctx_set_model(self.ctx.ptr, None))

    def close(self) -> None:
        if self.ptr:
            try:
                self.lib.si_ctx_set_model(self.ctx.ptr, None)
            except Exception:
                pass
            self.lib.si_model_destroy(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
