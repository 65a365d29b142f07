"""The learned potential: a BF16 MLP trained and evaluated on the B200 tensor cores (include/spo_mlp.h).

``Mlp`` wraps the C ABI; ``potential_features`` turns the points of a potential grid (the reference's
PotentialGrid layout, src/potential/potential_grid.hpp:21-37: V[itp + n_tp (irep + n_rep izr)],
itp = iphi + nphi itheta, izr = ir + nr iz) into network inputs. The exact potential values remain the
reference and the fallback: the network stands in for their evaluation on further points.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import capi

_EXPORTS = ["spo_mlp_create", "spo_mlp_destroy", "spo_mlp_last_error", "spo_mlp_parameter_count",
            "spo_mlp_get_parameters", "spo_mlp_set_parameters", "spo_mlp_input_width", "spo_mlp_predict",
            "spo_mlp_gradients", "spo_mlp_train"]


def _bind(lib):
    if getattr(lib, "_spo_mlp_bound", False):
        return lib
    h = ctypes.c_void_p
    fp = ctypes.POINTER(ctypes.c_float)
    dp = ctypes.POINTER(ctypes.c_double)
    lib.spo_mlp_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_ulonglong, ctypes.c_int,
                                   ctypes.POINTER(h)]
    lib.spo_mlp_destroy.argtypes = [h]
    lib.spo_mlp_last_error.argtypes = [h]
    lib.spo_mlp_last_error.restype = ctypes.c_char_p
    lib.spo_mlp_parameter_count.argtypes = [h, ctypes.POINTER(ctypes.c_longlong)]
    lib.spo_mlp_get_parameters.argtypes = [h, fp]
    lib.spo_mlp_set_parameters.argtypes = [h, fp]
    lib.spo_mlp_input_width.argtypes = [h, ctypes.POINTER(ctypes.c_int)]
    lib.spo_mlp_predict.argtypes = [h, fp, ctypes.c_longlong, fp]
    lib.spo_mlp_gradients.argtypes = [h, fp, fp, ctypes.c_longlong, dp, fp]
    lib.spo_mlp_train.argtypes = [h, fp, fp, ctypes.c_longlong, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                  ctypes.c_ulonglong, dp]
    for name in _EXPORTS:
        if name != "spo_mlp_last_error":
            getattr(lib, name).restype = ctypes.c_int
    lib._spo_mlp_bound = True
    return lib


def _f32(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


class Mlp:
    """n_in -> depth x width SiLU -> 1, BF16 products with FP32 accumulation on the tensor cores."""

    def __init__(self, n_in: int, width: int = 256, depth: int = 4, seed: int = 1, device: int = 0):
        self._lib = _bind(capi.lib())
        h = ctypes.c_void_p()
        st = self._lib.spo_mlp_create(n_in, width, depth, seed, device, ctypes.byref(h))
        if st != 0:
            raise capi.B200Error(st, self._lib.spo_mlp_last_error(None).decode())
        self._h = h
        self.n_in, self.width, self.depth = n_in, width, depth

    def _check(self, st):
        if st != 0:
            raise capi.B200Error(st, self._lib.spo_mlp_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self._lib.spo_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def input_width(self) -> int:
        n = ctypes.c_int()
        self._check(self._lib.spo_mlp_input_width(self._h, ctypes.byref(n)))
        return n.value

    def parameter_count(self) -> int:
        n = ctypes.c_longlong()
        self._check(self._lib.spo_mlp_parameter_count(self._h, ctypes.byref(n)))
        return n.value

    def get_parameters(self) -> np.ndarray:
        out = np.empty(self.parameter_count(), dtype=np.float32)
        self._check(self._lib.spo_mlp_get_parameters(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    def set_parameters(self, p: np.ndarray) -> None:
        p, pp = _f32(p)
        assert p.size == self.parameter_count()
        self._check(self._lib.spo_mlp_set_parameters(self._h, pp))

    def predict(self, x: np.ndarray) -> np.ndarray:
        x, xp = _f32(x)
        assert x.ndim == 2 and x.shape[1] == self.n_in
        y = np.empty(x.shape[0], dtype=np.float32)
        self._check(self._lib.spo_mlp_predict(self._h, xp, x.shape[0], y.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return y

    def gradients(self, x: np.ndarray, y: np.ndarray):
        x, xp = _f32(x)
        y, yp = _f32(y)
        g = np.empty(self.parameter_count(), dtype=np.float32)
        loss = ctypes.c_double()
        self._check(self._lib.spo_mlp_gradients(self._h, xp, yp, x.shape[0], ctypes.byref(loss),
                                                g.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return loss.value, g

    def train(self, x: np.ndarray, y: np.ndarray, epochs: int, batch: int = 4096, lr: float = 2e-3,
              seed: int = 7) -> float:
        x, xp = _f32(x)
        y, yp = _f32(y)
        loss = ctypes.c_double()
        self._check(self._lib.spo_mlp_train(self._h, xp, yp, x.shape[0], epochs, batch, lr, seed, ctypes.byref(loss)))
        return loss.value


def potential_features(z: np.ndarray, r: np.ndarray, nx: int, ny: int, theta: np.ndarray, phi: np.ndarray,
                       nz_potential: int) -> np.ndarray:
    """Inputs of every point of a potential grid without symmetry (n_rep = nx ny), in the grid's own
    order (itp fastest, then the (x, y) point, then izr = ir + nr iz): Z and r (as given), the (x, y)
    position through periodic functions of its fractional coordinates (u, v) = (ix / nx, iy / ny),
    and the orientation as the unit vector (sin th cos ph, sin th sin ph, cos th) with cos 2 ph, sin 2 ph.
    Returns float32 (n_points, 12)."""
    nr = len(r)
    th, ph = np.meshgrid(theta, phi, indexing="ij")                       # (nt, nphi), itp = iphi + nphi it
    ori = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th), np.cos(2 * ph), np.sin(2 * ph)],
                   axis=-1).reshape(-1, 5)
    ix, iy = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")      # ixy = iy + ny ix
    u, v = (ix / nx).ravel(), (iy / ny).ravel()
    two_pi = 2.0 * np.pi
    site = np.stack([np.cos(two_pi * u), np.sin(two_pi * u), np.cos(two_pi * v), np.sin(two_pi * v),
                     np.cos(two_pi * (u - v))], axis=-1)                   # (n_xy, 5)
    izr = np.arange(nz_potential * nr)
    zr = np.stack([np.asarray(z)[izr // nr], np.asarray(r)[izr % nr]], axis=-1)  # (n_zr, 2)
    n_tp, n_xy, n_zr = ori.shape[0], site.shape[0], zr.shape[0]
    f = np.empty((n_zr, n_xy, n_tp, 12), dtype=np.float32)
    f[..., 0:2] = zr[:, None, None, :]
    f[..., 2:7] = site[None, :, None, :]
    f[..., 7:12] = ori[None, None, :, :]
    return f.reshape(-1, 12)
