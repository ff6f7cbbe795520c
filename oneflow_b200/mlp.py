"""Python face of the warm-start MLP (ofg_mlp_* in include/oneflow_b200.h):
BF16 tensor-core training and inference kernels of libofg.so, with device
arrays held in torch tensors (plumbing only)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from .solver import OfgError, load_library


def _bind(L):
    if getattr(L, "_mlp_bound", False):
        return L
    L.ofg_mlp_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64, C.POINTER(C.c_void_p)]
    L.ofg_mlp_destroy.argtypes = [C.c_void_p]
    L.ofg_mlp_last_error.argtypes = [C.c_void_p]
    L.ofg_mlp_last_error.restype = C.c_char_p
    L.ofg_mlp_num_params.argtypes = [C.c_void_p]
    L.ofg_mlp_num_params.restype = C.c_int64
    L.ofg_mlp_get_params.argtypes = [C.c_void_p, C.c_void_p]
    L.ofg_mlp_set_params.argtypes = [C.c_void_p, C.c_void_p]
    L.ofg_mlp_predict.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]
    L.ofg_mlp_loss_grad.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
    L.ofg_mlp_train.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_float,
                                C.c_uint64, C.c_void_p]
    L._mlp_bound = True
    return L


def _dev(t):
    import torch
    assert t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()
    return C.c_void_p(t.data_ptr())


class MLP:
    """n_in -> depth x width (GELU) -> n_out, BF16 on the tensor cores."""

    def __init__(self, n_in: int, width: int, depth: int, n_out: int, seed: int = 0):
        self.L = _bind(load_library())
        self.shape = (n_in, width, depth, n_out)
        h = C.c_void_p()
        rc = self.L.ofg_mlp_create(n_in, width, depth, n_out, seed, C.byref(h))
        if rc != 0:
            raise OfgError(f"ofg_mlp_create failed ({rc})")
        self.h = h

    def _check(self, rc):
        if rc != 0:
            msg = self.L.ofg_mlp_last_error(self.h)
            raise OfgError(f"error {rc}: {msg.decode() if msg else ''}")

    def layer_shapes(self):
        n_in, w, d, n_out = self.shape
        dims = [n_in] + [w] * d + [n_out]
        return list(zip(dims[:-1], dims[1:]))

    def params(self) -> np.ndarray:
        out = np.empty(self.L.ofg_mlp_num_params(self.h), np.float32)
        self._check(self.L.ofg_mlp_get_params(self.h, out.ctypes.data_as(C.c_void_p)))
        return out

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        self._check(self.L.ofg_mlp_set_params(self.h, p.ctypes.data_as(C.c_void_p)))

    def unpack(self, flat: np.ndarray):
        """[(W [fan_in, fan_out], b [fan_out])] views of a flat parameter array"""
        out, o = [], 0
        for fi, fo in self.layer_shapes():
            W = flat[o:o + fi * fo].reshape(fi, fo); o += fi * fo
            b = flat[o:o + fo]; o += fo
            out.append((W, b))
        return out

    def predict(self, x):
        import torch
        y = torch.empty((x.shape[0], self.shape[3]), dtype=torch.float32, device=x.device)
        self._check(self.L.ofg_mlp_predict(self.h, _dev(x), x.shape[0], _dev(y)))
        return y

    def loss_grad(self, x, y):
        loss = C.c_float()
        g = np.empty(self.L.ofg_mlp_num_params(self.h), np.float32)
        self._check(self.L.ofg_mlp_loss_grad(self.h, _dev(x), _dev(y), x.shape[0], C.byref(loss),
                                             g.ctypes.data_as(C.c_void_p)))
        return float(loss.value), g

    def train(self, x, y, steps: int, batch: int = 8192, lr: float = 1e-3, seed: int = 0) -> np.ndarray:
        losses = np.zeros(steps, np.float32)
        self._check(self.L.ofg_mlp_train(self.h, _dev(x), _dev(y), x.shape[0], batch, steps, C.c_float(lr), seed,
                                          losses.ctypes.data_as(C.c_void_p)))
        return losses

    def close(self):
        if getattr(self, "h", None):
            self.L.ofg_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
