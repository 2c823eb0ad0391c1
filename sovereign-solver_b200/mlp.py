"""Python face of the learned warm start's network (pdhg_mlp_* in the C-ABI).

``Mlp(n_in, hidden, n_out)`` is a 2-hidden-layer ReLU network whose forward
and backward passes run on the B200 tensor cores (BF16 operands, FP32
accumulation) and whose training is Adam on FP32 master weights, all on the
device. There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import pdhg

_fp = C.POINTER(C.c_float)
_declared = False


def _lib() -> C.CDLL:
    global _declared
    L = pdhg.lib()
    if not _declared:
        L.pdhg_mlp_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                      C.POINTER(C.c_void_p)]
        L.pdhg_mlp_destroy.argtypes = [C.c_void_p]
        L.pdhg_mlp_last_error.argtypes = [C.c_void_p]
        L.pdhg_mlp_last_error.restype = C.c_char_p
        L.pdhg_mlp_param_count.argtypes = [C.c_void_p]
        L.pdhg_mlp_param_count.restype = C.c_int64
        L.pdhg_mlp_set_params.argtypes = [C.c_void_p, _fp]
        L.pdhg_mlp_get_params.argtypes = [C.c_void_p, _fp]
        L.pdhg_mlp_forward.argtypes = [C.c_void_p, C.c_int, _fp, _fp]
        L.pdhg_mlp_gradients.argtypes = [C.c_void_p, C.c_int, _fp, _fp, _fp, _fp]
        L.pdhg_mlp_train.argtypes = [C.c_void_p, C.c_int64, _fp, _fp, C.c_int, C.c_int,
                                     C.c_float, C.c_uint64, _fp]
        L.pdhg_mlp_adam_step.argtypes = [C.c_void_p, _fp, C.c_float]
        L.pdhg_gemm_bf16.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _fp, _fp, _fp, C.c_int,
                                     _fp]
        _declared = True
    return L


def _f(a: np.ndarray):
    return a.ctypes.data_as(_fp)


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


class Mlp:
    """n_in -> hidden -> hidden -> n_out ReLU network on one device."""

    def __init__(self, n_in: int, hidden: int, n_out: int, max_batch: int = 512,
                 device: int = 0) -> None:
        h = C.c_void_p()
        rc = _lib().pdhg_mlp_create(device, n_in, hidden, n_out, max_batch, C.byref(h))
        if rc != 0:
            raise pdhg.PdhgError(rc, "pdhg_mlp_create")
        self._h = h
        self.n_in, self.hidden, self.n_out, self.max_batch = n_in, hidden, n_out, max_batch

    def _check(self, rc: int, what: str) -> None:
        if rc != 0:
            raise pdhg.PdhgError(rc, f"{what} ({_lib().pdhg_mlp_last_error(self._h).decode()})")

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib().pdhg_mlp_destroy(self._h)
            self._h = None

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self) -> "Mlp":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    @property
    def param_count(self) -> int:
        return int(_lib().pdhg_mlp_param_count(self._h))

    def set_params(self, params: np.ndarray) -> None:
        p = _f32(params)
        assert p.size == self.param_count
        self._check(_lib().pdhg_mlp_set_params(self._h, _f(p)), "pdhg_mlp_set_params")

    def get_params(self) -> np.ndarray:
        p = np.zeros(self.param_count, dtype=np.float32)
        self._check(_lib().pdhg_mlp_get_params(self._h, _f(p)), "pdhg_mlp_get_params")
        return p

    def forward(self, x: np.ndarray) -> np.ndarray:
        """Any number of rows: padded to batches of a multiple of 8 internally."""
        x = _f32(x)
        rows = x.shape[0]
        out = np.zeros((rows, self.n_out), dtype=np.float32)
        step = self.max_batch
        for r0 in range(0, rows, step):
            xb = x[r0:r0 + step]
            b = xb.shape[0]
            bp = (b + 7) // 8 * 8
            if bp != b:
                xb = np.vstack([xb, np.zeros((bp - b, self.n_in), dtype=np.float32)])
            yb = np.zeros((bp, self.n_out), dtype=np.float32)
            self._check(_lib().pdhg_mlp_forward(self._h, bp, _f(_f32(xb)), _f(yb)),
                        "pdhg_mlp_forward")
            out[r0:r0 + b] = yb[:b]
        return out

    def gradients(self, x: np.ndarray, t: np.ndarray) -> tuple[np.ndarray, float]:
        x, t = _f32(x), _f32(t)
        g = np.zeros(self.param_count, dtype=np.float32)
        loss = C.c_float()
        self._check(_lib().pdhg_mlp_gradients(self._h, x.shape[0], _f(x), _f(t), _f(g),
                                              C.byref(loss)), "pdhg_mlp_gradients")
        return g, float(loss.value)

    def adam_step(self, grads: np.ndarray, lr: float = 1e-3) -> None:
        """One Adam step with the given gradients (parameter order): the update
        of data-parallel training, after the ranks averaged their gradients."""
        g = _f32(grads)
        assert g.size == self.param_count
        self._check(_lib().pdhg_mlp_adam_step(self._h, _f(g), lr), "pdhg_mlp_adam_step")

    def train(self, x: np.ndarray, t: np.ndarray, epochs: int, batch: int = 256,
              lr: float = 1e-3, seed: int = 0) -> np.ndarray:
        x, t = _f32(x), _f32(t)
        losses = np.zeros(max(epochs, 1), dtype=np.float32)
        self._check(_lib().pdhg_mlp_train(self._h, x.shape[0], _f(x), _f(t), epochs, batch,
                                          lr, seed, _f(losses)), "pdhg_mlp_train")
        return losses[:epochs]


def gemm_bf16(a: np.ndarray, b: np.ndarray, bias: np.ndarray | None = None, relu: bool = False,
              device: int = 0) -> np.ndarray:
    """C = A B^T (+ bias, ReLU) on the tensor cores (BF16 operands, FP32 sums)."""
    a, b = _f32(a), _f32(b)
    m, k = a.shape
    n = b.shape[0]
    c = np.zeros((m, n), dtype=np.float32)
    bi = _f32(bias) if bias is not None else None
    rc = _lib().pdhg_gemm_bf16(device, m, n, k, _f(a), _f(b),
                               _f(bi) if bi is not None else C.cast(None, _fp), int(relu), _f(c))
    if rc != 0:
        raise pdhg.PdhgError(rc, "pdhg_gemm_bf16")
    return c
