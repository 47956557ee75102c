"""Profile contraction Y = I . P with the cell and profile fixed (p6_ct_*).

A fixed cell and profile turn the pattern calculation of every replica into
one product: intensities I (replicas x reflections: the heights
scale * mult * Lp * |F|^2 / area of js/rietveld_core.js:881-886) times the
banded profile matrix P (reflections x points: the unit-height columns of
js/profile.js:1013-1090).  ``ContractionSession`` runs it on the B200 as a
split-BF16 tcgen05 product or as a plain FP32 CUDA-core product, with the
weighted chi^2 of every replica reduced in FP64.

``banded_problem`` builds the synthetic workload: reflections at sorted
random 2-theta, pseudo-Voigt columns of unit height with FWHM uniform in
[fwhm_lo, fwhm_hi] degrees truncated at +/- ``window`` FWHM, lognormal
intensities, and an observed pattern made from one more lognormal replica
with Poisson counts.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _lib
from ._lib import P6CtProblem, check

SPLIT_BF16 = 0
FP32 = 1
SPLIT3_BF16 = 2   # three bf16 parts, six products: limited by the tensor core's FP32 accumulation
FP32_DENSE = 3    # every reflection at every point on the CUDA cores (the reference's dense render)
METHOD_NAMES = {SPLIT_BF16: 'split-bf16', FP32: 'fp32-banded', SPLIT3_BF16: 'split3-bf16', FP32_DENSE: 'fp32-dense'}


@dataclass
class BandedProblem:
    tth: np.ndarray          # n_points
    centres: np.ndarray      # n_refl, sorted
    fwhm: np.ndarray         # n_refl
    eta: np.ndarray          # n_refl
    profile_t: np.ndarray    # n_points x n_refl float32 (P transposed)
    intensities: np.ndarray  # n_replicas x n_refl float32
    yobs: np.ndarray         # n_points float32
    w: np.ndarray            # n_points float32
    window: float


def pseudo_voigt(d: np.ndarray, fwhm: np.ndarray, eta: np.ndarray) -> np.ndarray:
    """Unit-height pseudo-Voigt: eta / (1 + 4 (d/G)^2) + (1 - eta) exp(-4 ln 2 (d/G)^2)."""
    u = (d / fwhm) ** 2
    return eta / (1.0 + 4.0 * u) + (1.0 - eta) * np.exp(-4.0 * np.log(2.0) * u)


def banded_problem(n_refl: int = 3000, n_points: int = 12000, n_replicas: int = 16384, tth0: float = 5.0,
                   step: float = 0.01, fwhm_lo: float = 0.05, fwhm_hi: float = 0.3, window: float = 20.0,
                   sigma: float = 1.5, counts: float = 100.0, seed: int = 1) -> BandedProblem:
    rng = np.random.default_rng(seed)
    tth = tth0 + step * np.arange(n_points, dtype=np.float64)
    span = tth[-1] - tth[0]
    centres = np.sort(rng.uniform(tth[0] + 0.01 * span, tth[-1] - 0.01 * span, n_refl))
    fwhm = rng.uniform(fwhm_lo, fwhm_hi, n_refl)
    eta = rng.uniform(0.0, 1.0, n_refl)
    pt = np.zeros((n_points, n_refl), dtype=np.float32)
    for r in range(n_refl):
        half = window * fwhm[r]
        lo = int(np.searchsorted(tth, centres[r] - half, 'left'))
        hi = int(np.searchsorted(tth, centres[r] + half, 'right'))
        if hi > lo:
            pt[lo:hi, r] = pseudo_voigt(tth[lo:hi] - centres[r], fwhm[r], eta[r])
    intens = rng.lognormal(0.0, sigma, (n_replicas, n_refl)).astype(np.float32)
    truth = rng.lognormal(0.0, sigma, n_refl)
    ytrue = pt.astype(np.float64) @ truth
    yobs = rng.poisson(np.maximum(ytrue, 0) * counts) / counts
    w = 1.0 / np.maximum(yobs, 1.0 / counts)
    return BandedProblem(tth, centres, fwhm, eta, pt, intens, yobs.astype(np.float32), w.astype(np.float32), window)


class ContractionSession:
    """p6_ct_create ... p6_ct_destroy."""

    def __init__(self, prob: BandedProblem, max_replicas: Optional[int] = None, device: int = 0):
        self.lib = _lib.load()
        self.prob = prob
        self.n_points, self.n_refl = prob.profile_t.shape
        self.max_replicas = int(max_replicas or len(prob.intensities))
        self._keep = [np.ascontiguousarray(prob.profile_t, dtype=np.float32),
                      np.ascontiguousarray(prob.yobs, dtype=np.float32),
                      np.ascontiguousarray(prob.w, dtype=np.float32)]
        pr = P6CtProblem()
        pr.n_refl = self.n_refl
        pr.n_points = self.n_points
        pr.max_replicas = self.max_replicas
        pr.profile_t = self._keep[0].ctypes.data
        pr.yobs = self._keep[1].ctypes.data
        pr.w = self._keep[2].ctypes.data
        h = C.c_void_p()
        check(self.lib.p6_ct_create(C.byref(pr), int(device), C.byref(h)))
        self.h = h
        self.m = 0

    def close(self):
        if getattr(self, 'h', None):
            self.lib.p6_ct_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_intensities(self, intensities: np.ndarray):
        a = np.ascontiguousarray(intensities, dtype=np.float32)
        self._intens = a
        check(self.lib.p6_ct_set_intensities(self.h, a.ctypes.data, len(a)))
        self.m = len(a)

    def evaluate(self, method: int = SPLIT_BF16, store_pattern: bool = False):
        check(self.lib.p6_ct_evaluate(self.h, int(method), 1 if store_pattern else 0))

    def read(self, pattern: bool = False):
        chi = np.zeros(self.m)
        y = np.zeros((self.m, self.n_points), dtype=np.float32) if pattern else None
        check(self.lib.p6_ct_read(self.h, chi.ctypes.data, None if y is None else y.ctypes.data))
        return (chi, y) if pattern else chi

    def run(self, intensities: np.ndarray, method: int = SPLIT_BF16, pattern: bool = False):
        self.set_intensities(intensities)
        self.evaluate(method, pattern)
        return self.read(pattern)

    def run_host(self, intensities: np.ndarray, method: int = SPLIT_BF16) -> np.ndarray:
        a = np.ascontiguousarray(intensities, dtype=np.float32)
        chi = np.zeros(len(a))
        check(self.lib.p6_ct_run_host(self.h, a.ctypes.data, len(a), int(method), chi.ctypes.data))
        self.m = len(a)
        return chi

    def set_fitted(self, on: bool = True):
        """chi^2 at each replica's best scale instead of the intensities as given."""
        check(self.lib.p6_ct_set_fitted(self.h, 1 if on else 0))

    def read_scale(self) -> np.ndarray:
        s = np.zeros(self.m)
        check(self.lib.p6_ct_read_scale(self.h, s.ctypes.data))
        return s

    def synchronize(self):
        check(self.lib.p6_ct_synchronize(self.h))

    def last_ms(self) -> float:
        v = C.c_float()
        check(self.lib.p6_ct_last_ms(self.h, C.byref(v)))
        return v.value

    def query(self) -> dict:
        kb, c128, nt, ln = C.c_longlong(), C.c_longlong(), C.c_int(), C.c_longlong()
        check(self.lib.p6_ct_query(self.h, C.byref(kb), C.byref(c128), C.byref(nt), C.byref(ln)))
        return {'band_kblocks': kb.value, 'band_cols128': c128.value, 'n_tiles': nt.value, 'launches': ln.value}
