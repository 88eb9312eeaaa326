"""The learned SU(3) Metropolis proposal (no reference counterpart).

A ``ProposalModel`` is a small network on the device that maps sixteen
gauge-invariant features of a link's staple sum to eight generator logits
and an angle scale (include/ym_learned.h has the exact definition).  It is
trained on configurations the plain sampler generates, by the engine's own
tensor-core forward and backward kernels, to maximise the expected squared
change of the local action in one hit; ``Ensemble`` chains in two-row binary32 storage are then
swept with it.  The proposal depends on the staple only, so it is symmetric
and the exact accept/reject keeps detailed balance; plain Metropolis
(``Ensemble.metropolis_sweeps``) stays the reference sampler it is judged
against through the reference's autocorrelation estimator
(su2_ensemble.rs:375-463).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import lib
from .ensemble import Ensemble
from .errors import check

N_FEATURES = 16
N_OUTPUTS = 16
N_PARAMS = 6288
OFFSETS = {"W1": 0, "b1": 1024, "W2": 1088, "b2": 5184, "W3": 5248, "b3": 6272}
SCALE_MIN, SCALE_MAX = 0.05, 2.5
GENERATOR_FLOOR = 0.5


def _fp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class ProposalModel:
    """Parameters, Adam state and BF16 weight image on one device."""

    def __init__(self, device: int = 0, seed: int = 0x4C50524F504F5341, initial_scale: float = 0.3):
        h = C.c_void_p()
        check(lib().ym_model_create(int(device), int(seed) & (2 ** 64 - 1), float(initial_scale),
                                    C.byref(h)), "model_create")
        self._h = h
        self.device = device

    def close(self) -> None:
        if getattr(self, "_h", None):
            check(lib().ym_model_destroy(self._h), "model_destroy")
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
    def params(self) -> np.ndarray:
        out = np.zeros(N_PARAMS, np.float32)
        check(lib().ym_model_get_params(self._h, _fp(out)), "model_get_params")
        return out

    @params.setter
    def params(self, value) -> None:
        p = np.ascontiguousarray(value, np.float32).reshape(N_PARAMS)
        check(lib().ym_model_set_params(self._h, _fp(p)), "model_set_params")

    def forward(self, features) -> np.ndarray:
        """Network outputs [n, 16] (tensor-core forward)."""
        x = np.ascontiguousarray(features, np.float32).reshape(-1, N_FEATURES)
        y = np.zeros((x.shape[0], N_OUTPUTS), np.float32)
        check(lib().ym_model_forward(self._h, _fp(x), x.shape[0], _fp(y)), "model_forward")
        return y

    def gradient(self, features, m, beta):
        """(mean objective, gradient of -mean objective) over records."""
        x = np.ascontiguousarray(features, np.float32).reshape(-1, N_FEATURES)
        mm = np.ascontiguousarray(m, np.float32).reshape(-1, 18)
        b = np.ascontiguousarray(np.broadcast_to(np.asarray(beta, np.float64), (x.shape[0],)).copy())
        g = np.zeros(N_PARAMS, np.float32)
        obj = C.c_double()
        check(lib().ym_model_gradient(self._h, _fp(x), _fp(mm), _dp(b), x.shape[0], C.byref(obj),
                                      _fp(g)), "model_gradient")
        return obj.value, g

    def train(self, ens: Ensemble, n_steps: int, sweeps_per_step: int = 1,
              plain_angle: float = 0.3, lr: float = 2e-3) -> np.ndarray:
        """On-device training; returns the objective of every step."""
        hist = np.zeros(max(int(n_steps), 1), np.float64)
        check(lib().ym_model_train(self._h, ens.handle, int(n_steps), int(sweeps_per_step),
                                   float(plain_angle), float(lr), _dp(hist)), "model_train")
        return hist[:n_steps]

    def sweeps(self, ens: Ensemble, n_sweeps: int = 1) -> None:
        check(lib().ym_su3_learned_sweeps(ens.handle, self._h, int(n_sweeps)), "su3_learned_sweeps")

    def measured_sweeps(self, ens: Ensemble, n_measurements: int,
                        sweeps_per_measurement: int = 1) -> np.ndarray:
        out = np.zeros((n_measurements, ens.n_chains), np.float64)
        check(lib().ym_su3_learned_measured_sweeps(ens.handle, self._h, int(n_measurements),
                                                   int(sweeps_per_measurement), _dp(out)),
              "su3_learned_measured_sweeps")
        return out


def records(ens: Ensemble, parity: int, mu: int):
    """Training records of one sub-sweep: features [n,16], M = U A [n,18], beta [n]."""
    n = C.c_int64()
    check(lib().ym_learned_records(ens.handle, int(parity), int(mu), None, None, None, C.byref(n)),
          "learned_records")
    f = np.zeros((n.value, N_FEATURES), np.float32)
    m = np.zeros((n.value, 18), np.float32)
    b = np.zeros(n.value, np.float64)
    check(lib().ym_learned_records(ens.handle, int(parity), int(mu), _fp(f), _fp(m), _dp(b),
                                   C.byref(n)), "learned_records")
    return f, m, b


def proposal(outputs):
    """Generator probabilities [n, 8] and angle half widths [n] from outputs."""
    y = np.asarray(outputs, np.float64).reshape(-1, N_OUTPUTS)
    z = np.exp(y[:, :8] - y[:, :8].max(1, keepdims=True))
    p = GENERATOR_FLOOR / 8 + (1 - GENERATOR_FLOOR) * z / z.sum(1, keepdims=True)
    s = SCALE_MIN + (SCALE_MAX - SCALE_MIN) / (1.0 + np.exp(-y[:, 8]))
    return p, s
