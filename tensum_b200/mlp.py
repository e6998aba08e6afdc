"""ctypes binding of the surrogate network (tg_mlp_* in include/tensum_gpu.h)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import gpu

H = 64
_bound = False


def _lib():
    global _bound
    L = gpu.load()
    if not _bound:
        vp, i, fp = C.c_void_p, C.c_int, C.POINTER(C.c_float)
        L.tg_mlp_create.argtypes = [i, i, C.c_ulonglong, C.POINTER(vp)]
        L.tg_mlp_destroy.argtypes = [vp]
        L.tg_mlp_last_error.argtypes = [vp]
        L.tg_mlp_last_error.restype = C.c_char_p
        L.tg_mlp_n_params.argtypes = [vp]
        L.tg_mlp_n_params.restype = i
        L.tg_mlp_get_params.argtypes = [vp, fp]
        L.tg_mlp_set_params.argtypes = [vp, fp]
        L.tg_mlp_loss_grad.argtypes = [vp, fp, fp, i, fp, fp]
        L.tg_mlp_train.argtypes = [vp, fp, fp, i, i, i, C.c_float, fp]
        L.tg_mlp_predict.argtypes = [vp, vp, i, vp, i, i]
        for n in ("tg_mlp_create", "tg_mlp_destroy", "tg_mlp_get_params", "tg_mlp_set_params", "tg_mlp_loss_grad",
                  "tg_mlp_train", "tg_mlp_predict"):
            getattr(L, n).restype = i
        _bound = True
    return L


def _f(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def n_params(din: int, dout: int) -> int:
    return H * din + H + 2 * (H * H + H) + dout * H + dout


class MLP:
    """din -> 64 -> 64 -> 64 -> dout GELU network on the GPU, with input and
    output standardisation kept on the host (fitted on the training set)."""

    def __init__(self, din: int, dout: int, seed: int = 0):
        self.L = _lib()
        self.din, self.dout = din, dout
        h = C.c_void_p()
        st = self.L.tg_mlp_create(din, dout, seed, C.byref(h))
        if st != 0:
            raise gpu.TensumError(st, self.L.tg_mlp_last_error(None).decode())
        self.h = h
        self.np = self.L.tg_mlp_n_params(h)
        self.xm = np.zeros(din); self.xs = np.ones(din)
        self.ym = np.zeros(dout); self.ys = np.ones(dout)

    def __del__(self):
        try:
            if getattr(self, "h", None):
                self.L.tg_mlp_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def _chk(self, st):
        if st != 0:
            raise gpu.TensumError(st, self.L.tg_mlp_last_error(self.h).decode())

    @property
    def params(self) -> np.ndarray:
        out = np.empty(self.np, np.float32)
        self._chk(self.L.tg_mlp_get_params(self.h, _f(out)))
        return out

    @params.setter
    def params(self, theta):
        theta = np.ascontiguousarray(theta, np.float32)
        assert theta.size == self.np
        self._chk(self.L.tg_mlp_set_params(self.h, _f(theta)))

    def loss_grad(self, X, T):
        """Loss and gradient of one batch in network units (no standardisation)."""
        X = np.ascontiguousarray(X, np.float32)
        T = np.ascontiguousarray(T, np.float32)
        loss = np.empty(1, np.float32)
        g = np.empty(self.np, np.float32)
        self._chk(self.L.tg_mlp_loss_grad(self.h, _f(X), _f(T), X.shape[0], _f(loss), _f(g)))
        return float(loss[0]), g

    def fit(self, X, Y, epochs: int = 200, batch: int = 64, lr: float = 3e-3) -> np.ndarray:
        """Standardise inputs and outputs on this set, then train; returns the per-epoch losses."""
        X = np.asarray(X, np.float64)
        Y = np.asarray(Y, np.float64)
        self.xm, self.xs = X.mean(axis=0), X.std(axis=0) + 1e-12
        self.ym, self.ys = Y.mean(axis=0), Y.std(axis=0) + 1e-300
        Xn = np.ascontiguousarray((X - self.xm) / self.xs, np.float32)
        Yn = np.ascontiguousarray((Y - self.ym) / self.ys, np.float32)
        losses = np.empty(epochs, np.float32)
        self._chk(self.L.tg_mlp_train(self.h, _f(Xn), _f(Yn), Xn.shape[0], epochs, batch, lr, _f(losses)))
        return losses

    def raw_predict(self, X, precision: int = 0) -> np.ndarray:
        X = np.ascontiguousarray(X, np.float32)
        Y = np.empty((X.shape[0], self.dout), np.float32)
        self._chk(self.L.tg_mlp_predict(self.h, X.ctypes.data, X.shape[0], Y.ctypes.data, precision, 0))
        return Y

    def predict(self, X, precision: int = 1) -> np.ndarray:
        """Surrogate QoIs for inputs X (physical units); precision 1 = BF16 tensor cores."""
        Xn = (np.asarray(X, np.float64) - self.xm) / self.xs
        return self.raw_predict(Xn, precision).astype(np.float64) * self.ys + self.ym
