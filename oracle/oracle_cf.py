"""ORACLE -- test infrastructure, not product code.

FP64 restatement of one charge-flipping cycle on a powder reflection model,
in the order js/charge_flipping_worker.js:2353-2395 dispatches the kernels of
charge_flipping.wgsl:

  F -> rho          cfEncodeFFT inverse (fft_stage, scale_inverse; :182-260)
  delta             reduce_moments / finalize_moments (:281-334):
                    delta_sigma * sqrt(max(0, <Re rho^2> - <Re rho>^2))
  flip              flip (:336-346): Re rho < delta -> -Re rho, Im rho = 0
  rho -> F          cfEncodeFFT forward
  R                 reduce_rfactor / finalize_rfactor (:552-583, :621-644):
                    sum |sqrt(I_calc(cluster)) - sqrt(I_obs)| / sum sqrt(I_obs)
  repartition       (:413-452) cluster intensity shared by calculated intensities
  symmetrize        (:367-404) orbit average through the members' phase factors,
                    mixed with weight sym_lambda (skipped at sym_lambda <= 0)
  constrain         (:463-527) |F| = sqrt(target / count), or the quarter-turn
                    of a weak orbit; a collapsed member restarts on a random phase
  zero_absent, zero_dc (:531-546)
  keep_best, commit_best (:598-619): the grid is kept when R < best R

The FFTs are numpy's (complex128).  The random restart draws the same
Philox4x32-10 word the device does (counter (member, 0x43465246, 0, 0), key
(seed, 0x52535452)), through the C oracle's ``p6o_philox``.  Grid index
h + k n + l n^2 is numpy's C order of an (n, n, n) array indexed [l, k, h].
"""
from __future__ import annotations

import math

import numpy as np

IDX_MASK = 0x7FFFFFFF
CONJ_BIT = 0x80000000


def philox_u01(member: int, seed: int) -> float:
    from oracle import oracle as O
    lib = O.load()
    ctr = np.array([member & 0xFFFFFFFF, 0x43465246, 0, 0], np.uint32)
    key = np.array([seed & 0xFFFFFFFF, 0x52535452], np.uint32)
    out = np.zeros(4, np.uint32)
    lib.p6o_philox(ctr.ctypes.data, key.ctypes.data, out.ctypes.data)
    return float(int(out[0]) >> 8) / 16777216.0


class CfState:
    """One trial: the complex F grid (flat, h + k n + l n^2), the best grid and
    best R, and its settings."""

    def __init__(self, model: dict, grid: np.ndarray, delta_sigma: float, sym_lambda: float, seed: int,
                 weak=None):
        self.m = model
        self.n = int(model['N'])
        g = np.asarray(grid, np.float64)
        self.F = g[0::2] + 1j * g[1::2]
        self.best = self.F.copy()
        self.best_r = math.inf
        self.delta_sigma = float(delta_sigma)
        self.sym_lambda = float(sym_lambda)
        self.seed = int(seed)
        self.weak = None if weak is None else np.asarray(weak, bool)
        self.last_rho = None
        self.last_delta = None
        self.pre_mag = None      # per grid point: |F| just before the amplitude constraint (NaN elsewhere)
        self.fft_max = 0.0       # max |F| out of the forward transform

    def cycle(self) -> float:
        m, n = self.m, self.n
        rho = np.fft.ifftn(self.F.reshape(n, n, n)).ravel()
        re = rho.real
        mean = re.mean()
        var = max(0.0, float((re * re).mean() - mean * mean))
        delta = self.delta_sigma * math.sqrt(var)
        self.last_rho, self.last_delta = re.copy(), delta
        flipped = np.where(re < delta, -re, re)
        F = np.fft.fftn(flipped.reshape(n, n, n)).ravel()
        self.fft_max = float(np.abs(F).max())
        self.pre_mag = np.full(F.size, np.nan)
        idx_all = m['orbit_idx']
        ph = m['phase'].astype(np.float64)
        num = den = 0.0
        lam = min(1.0, max(0.0, self.sym_lambda))
        for c in range(m['n_clusters']):
            o0, no = int(m['cluster_orbit_start'][c]), int(m['cluster_n_orbits'][c])
            obs = float(m['cluster_obs_i'][c])
            orbits = [(int(m['orbit_start'][o]), int(m['orbit_count'][o])) for o in range(o0, o0 + no)]
            sums = []
            for st, cnt in orbits:
                idx = idx_all[st:st + cnt] & IDX_MASK
                sums.append(float(np.sum(np.abs(F[idx]) ** 2)))
            total = sum(sums)
            members = sum(cnt for _, cnt in orbits)
            t = math.sqrt(max(0.0, obs))
            num += abs(math.sqrt(max(0.0, total)) - t)
            den += t
            for j, (st, cnt) in enumerate(orbits):
                o = o0 + j
                target = sums[j] * (obs / total) if total > 1e-20 else obs * cnt / members
                words = idx_all[st:st + cnt].astype(np.int64)
                idx = words & IDX_MASK
                conj = (words & CONJ_BIT) != 0
                cr, ci = ph[2 * st:2 * (st + cnt):2], ph[2 * st + 1:2 * (st + cnt):2]
                if self.sym_lambda > 0 and cnt >= 2:
                    a, b = F[idx].real, np.where(conj, -F[idx].imag, F[idx].imag)
                    sr = float(np.sum(a * cr + b * ci)) / cnt
                    si = float(np.sum(b * cr - a * ci)) / cnt
                    na = sr * cr - si * ci
                    nb = np.where(conj, -(sr * ci + si * cr), sr * ci + si * cr)
                    F[idx] = F[idx] * (1 - lam) + (na + 1j * nb) * lam
                if self.weak is not None and self.weak[o]:
                    h, k, l = idx % n, (idx // n) % n, idx // (n * n)
                    mate = (n - h) % n + ((n - k) % n) * n + ((n - l) % n) * n * n
                    f = F[idx]
                    F[idx] = np.where(idx > mate, f.imag - 1j * f.real, -f.imag + 1j * f.real)
                else:
                    amp = math.sqrt(max(0.0, target) / cnt)
                    f = F[idx]
                    mag = np.abs(f)
                    self.pre_mag[idx] = mag
                    out = np.empty_like(f)
                    live = mag > 1e-20
                    out[live] = f[live] * (amp / mag[live])
                    for q in np.nonzero(~live)[0]:
                        ang = 2 * math.pi * philox_u01(st + int(q), self.seed)
                        out[q] = amp * (math.cos(ang) + 1j * math.sin(ang))
                    F[idx] = out
        absent = m['orbit_idx'][m['absent_start']:m['absent_start'] + m['absent_count']] & IDX_MASK
        F[absent] = 0
        F[0] = 0
        R = num / den if den > 0 else math.nan
        if den > 0 and R < self.best_r:
            self.best_r = R
            self.best = F.copy()
        self.F = F
        return R

    def tolerance(self, base: float, fft_rel: float) -> np.ndarray:
        """Per grid point bound on |F_device - F_oracle| after the last cycle:
        ``base`` plus, for a constrained member, the phase error the forward
        transform's error (``fft_rel`` of its largest |F|) causes when the
        member is rescaled from magnitude |F_pre| to its target: |F| times
        min(2, 4 fft_rel max|F| / |F_pre|).  Small |F_pre| make the constraint
        ill-conditioned; everything else is held to ``base``."""
        amp = np.abs(self.F)
        pm = self.pre_mag
        cond = np.where(np.isfinite(pm), amp * np.minimum(2.0, 4 * fft_rel * self.fft_max / np.maximum(
            np.nan_to_num(pm, nan=1.0), 1e-300)), 0.0)
        return base + cond

    def ambiguous(self, band: float) -> int:
        """Points of the last flip within band * sigma of the threshold: where
        the FP32 device may decide the other way."""
        if self.last_rho is None:
            return 0
        sigma = self.last_delta / self.delta_sigma if self.delta_sigma else 0.0
        return int(np.sum(np.abs(self.last_rho - self.last_delta) < band * max(sigma, 1e-300)))

    def grid(self, which: str = 'current') -> np.ndarray:
        F = self.F if which == 'current' else self.best
        out = np.empty(2 * F.size)
        out[0::2], out[1::2] = F.real, F.imag
        return out
