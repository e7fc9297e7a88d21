"""Learned settling velocity: host side of the f3d_mlp_* C ABI.

A 5 -> 64 -> 64 -> 1 tanh network replaces the fixed-point drag-law solve of
phys_get_vset_point (mod_Phys.F90:757-954) inside phys_get_vset
(mod_Phys.F90:673-740).  Samples are drawn and labelled on the device by the
model's own iteration, the network is trained by the library's forward,
backward and Adam kernels, and inference runs its 64 x 64 layer on the
tensor cores.  Points outside the envelope take the iteration itself.

Typical use (the defaults are the envelope of the learned-vset workload):

    s = SettlingSurrogate(model=2)
    s.generate(1 << 20)
    s.train()
    v = s.predict(d, rhop, psi, rhoa, mu)
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib

NPARAMS = 4609
# diameter 1 um - 2 mm, particle density 800-3000 kg/m3, sphericity 0.5-1,
# air density 0.2-1.3 kg/m3, air viscosity 1.4e-5-1.8e-5 Pa s
DEFAULT_ENVELOPE = (1e-6, 2e-3, 800.0, 3000.0, 0.5, 1.0, 0.2, 1.3, 1.4e-5, 1.8e-5)
_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class SettlingSurrogate:
    """Owner of one f3d_mlp handle (parameters, samples, optimiser state)."""

    def __init__(self, model=2, envelope=DEFAULT_ENVELOPE, margin=0.08, seed=0, device=0):
        env = _d(envelope)
        if env.shape != (10,):
            raise ValueError("envelope: 10 numbers (lo, hi) x (d, rhop, psi, rhoa, visc)")
        self.model = int(model)
        self.envelope = env
        h = C.c_void_p()
        check(lib().f3d_mlp_create(self.model, env.ctypes.data_as(_dp), float(margin), int(seed),
                                   int(device), C.byref(h)), "f3d_mlp_create")
        self._h = h

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            lib().f3d_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- data and training -------------------------------------------------
    def generate(self, nsamples=1 << 20, seed=1) -> int:
        nf = C.c_longlong(0)
        check(lib().f3d_mlp_generate(self._h, int(nsamples), int(seed), C.byref(nf)), "f3d_mlp_generate")
        return nf.value

    def samples(self, first, n):
        raw = np.empty((n, 5), np.float64)
        rec = np.empty((n, 8), np.float32)
        check(lib().f3d_mlp_get_samples(self._h, int(first), int(n), raw.ctypes.data_as(_dp),
                                        rec.ctypes.data_as(_fp)), "f3d_mlp_get_samples")
        return raw, rec

    def train(self, steps=200000, batch=8192, lr_max=5e-3, lr_min=1e-5, seed=2):
        """Returns (loss per step, device milliseconds)."""
        loss = np.empty(max(steps, 1), np.float32)
        ms = C.c_float(0.0)
        check(lib().f3d_mlp_train(self._h, int(steps), int(batch), float(lr_max), float(lr_min), int(seed),
                                  loss.ctypes.data_as(_fp), C.byref(ms)), "f3d_mlp_train")
        return loss[:steps], ms.value

    def gradient(self, features, targets):
        f = np.ascontiguousarray(features, dtype=np.float32).reshape(-1, 5)
        t = np.ascontiguousarray(targets, dtype=np.float32).reshape(-1)
        g = np.empty(NPARAMS, np.float32)
        loss = C.c_float(0.0)
        check(lib().f3d_mlp_gradient(self._h, len(t), f.ctypes.data_as(_fp), t.ctypes.data_as(_fp),
                                     g.ctypes.data_as(_fp), C.byref(loss)), "f3d_mlp_gradient")
        return g, loss.value

    @property
    def params(self) -> np.ndarray:
        p = np.empty(NPARAMS, np.float32)
        check(lib().f3d_mlp_get_params(self._h, p.ctypes.data_as(_fp)), "f3d_mlp_get_params")
        return p

    @params.setter
    def params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.shape != (NPARAMS,):
            raise ValueError(f"expected {NPARAMS} parameters")
        check(lib().f3d_mlp_set_params(self._h, p.ctypes.data_as(_fp)), "f3d_mlp_set_params")

    def norm(self) -> np.ndarray:
        out = np.empty(19, np.float64)
        check(lib().f3d_mlp_get_norm(self._h, out.ctypes.data_as(_dp)), "f3d_mlp_get_norm")
        return out

    # -- inference ---------------------------------------------------------
    def predict(self, diam, rhop, psi, rhoa, visc, refine=0):
        """Settling velocity per point and the mask of points the surrogate
        answered (the others took the iteration)."""
        arrs = [_d(a).reshape(-1) for a in (diam, rhop, psi, rhoa, visc)]
        n = len(arrs[0])
        v = np.empty(n, np.float64)
        used = np.empty(n, np.int32)
        check(lib().f3d_mlp_predict(self._h, n, *[a.ctypes.data_as(_dp) for a in arrs], int(refine),
                                    v.ctypes.data_as(_dp), used.ctypes.data_as(_ip)), "f3d_mlp_predict")
        return v, used.astype(bool)

    def last_ms(self) -> float:
        ms = C.c_float(0.0)
        check(lib().f3d_mlp_last_ms(self._h, C.byref(ms)), "f3d_mlp_last_ms")
        return ms.value


def trained_surrogate(model=2, nsamples=1 << 20, steps=200000, batch=8192, lr_max=5e-3, seed=0, device=0):
    """Generate, train and return a surrogate with the default envelope
    (defaults: 2^20 samples, 200k Adam steps of 8192 samples, a few seconds
    on one GPU)."""
    s = SettlingSurrogate(model=model, seed=seed, device=device)
    s.generate(nsamples, seed=seed + 1)
    loss, ms = s.train(steps=steps, batch=batch, lr_max=lr_max, seed=seed + 2)
    s.train_loss, s.train_ms = loss, ms
    return s
