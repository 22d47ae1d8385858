"""The learned constitutive closure (include/retainwall.h, rw_mlp_*): a small perceptron
that predicts the objective part of the HypoCS stress rate, trained and evaluated on the
tensor cores by the native library."""
from __future__ import annotations

import ctypes as ct
from typing import Optional, Tuple

import numpy as np

from ._lib import RwError, lib

IN, OUT, NPARAM = 16, 6, 13958


def _check(status: int, what: str, h=None) -> None:
    if status != 0:
        d = lib().rw_mlp_last_error(h)
        raise RwError(status, what, d.decode() if d else "")


def _f32(a, shape_tail: int) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float32)
    if a.ndim != 2 or a.shape[1] != shape_tail:
        raise ValueError(f"expected an (n, {shape_tail}) array")
    return a


class Mlp:
    """16-64-64-64-64-6 SiLU perceptron with BF16 weights on one GPU."""

    def __init__(self, device: int = 0, seed: int = 0, sample_capacity: int = 0):
        h = ct.c_void_p()
        _check(lib().rw_mlp_create(device, seed, sample_capacity, ct.byref(h)), "rw_mlp_create")
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().rw_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def params(self) -> np.ndarray:
        p = np.empty(NPARAM, np.float32)
        _check(lib().rw_mlp_get_params(self._h, p.ctypes.data, NPARAM), "rw_mlp_get_params", self._h)
        return p

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.shape != (NPARAM,):
            raise ValueError(f"expected {NPARAM} parameters")
        _check(lib().rw_mlp_set_params(self._h, p.ctypes.data, NPARAM), "rw_mlp_set_params", self._h)

    def forward(self, x) -> np.ndarray:
        x = _f32(x, IN)
        y = np.empty((len(x), OUT), np.float32)
        _check(lib().rw_mlp_forward(self._h, x.ctypes.data, len(x), y.ctypes.data), "rw_mlp_forward", self._h)
        return y

    def grad(self, x, t) -> Tuple[float, np.ndarray]:
        x, t = _f32(x, IN), _f32(t, OUT)
        g = np.empty(NPARAM, np.float32)
        loss = ct.c_double()
        _check(lib().rw_mlp_grad(self._h, x.ctypes.data, t.ctypes.data, len(x), ct.byref(loss), g.ctypes.data),
               "rw_mlp_grad", self._h)
        return loss.value, g

    def add_samples(self, x, t) -> None:
        x, t = _f32(x, IN), _f32(t, OUT)
        _check(lib().rw_mlp_add_samples(self._h, x.ctypes.data, t.ctypes.data, len(x)), "rw_mlp_add_samples",
               self._h)

    def sample_count(self) -> int:
        c = ct.c_int64()
        _check(lib().rw_mlp_samples(self._h, ct.byref(c), None, None, 0), "rw_mlp_samples", self._h)
        return c.value

    def samples(self, n: Optional[int] = None):
        n = self.sample_count() if n is None else n
        x = np.empty((n, IN), np.float32)
        t = np.empty((n, OUT), np.float32)
        c = ct.c_int64()
        _check(lib().rw_mlp_samples(self._h, ct.byref(c), x.ctypes.data, t.ctypes.data, n), "rw_mlp_samples",
               self._h)
        return x, t

    def clear_samples(self) -> None:
        _check(lib().rw_mlp_clear_samples(self._h), "rw_mlp_clear_samples", self._h)

    def train(self, epochs: int, batch: int = 19456, lr: float = 1e-3, seed: int = 0) -> float:
        loss = ct.c_double()
        _check(lib().rw_mlp_train(self._h, epochs, batch, lr, seed, ct.byref(loss)), "rw_mlp_train", self._h)
        return loss.value

    def collect(self, sim, stride: int = 1, augment=None, seed: int = 0) -> int:
        """Appends samples from a LoquatSph's current state (every stride-th soil
        particle); ``augment`` = (phi min, phi max [deg], e0 min, e0 max) draws each
        sample's material from those ranges.  Returns how many were kept."""
        n = ct.c_int64()
        aug = None
        if augment is not None:
            arr = (ct.c_double * 4)(*augment)
            aug = ct.cast(arr, ct.c_void_p)
        check_ctx = lib().rw_mlp_collect(self._h, sim.handle, stride, aug, seed, ct.byref(n))
        if check_ctx != 0:
            d = lib().rw_last_error(sim.handle)
            raise RwError(check_ctx, "rw_mlp_collect", d.decode() if d else "")
        return n.value

    def feature_ranges(self):
        lo = np.empty(IN, np.float32)
        hi = np.empty(IN, np.float32)
        tm = np.empty(1, np.float32)
        _check(lib().rw_mlp_feature_ranges(self._h, lo.ctypes.data, hi.ctypes.data, tm.ctypes.data),
               "rw_mlp_feature_ranges", self._h)
        return lo, hi, float(tm[0])


# Material ranges of the learned closure's training set: friction angle [deg] and
# initial void ratio.
TRAIN_RANGES = (28.0, 40.0, 0.55, 0.80)


def training_run(net: Mlp, case, steps: int, every: int, stride: int = 1, device: int = 0, augment=TRAIN_RANGES,
                 seed: int = 0) -> int:
    """Runs the plain step on ``case`` for ``steps`` steps and stores samples in ``net``
    every ``every`` steps (materials drawn from ``augment``, None: the case's own);
    returns the number of samples added."""
    from .sph import LoquatSph

    sim = LoquatSph(case=case, device=device)
    added = 0
    for k, s in enumerate(range(0, steps, every)):
        sim.step(min(every, steps - s))
        added += net.collect(sim, stride, augment, seed * 1000003 + k)
    sim.close()
    return added
