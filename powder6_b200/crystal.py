"""Cell geometry used on the trial-evaluation path.

Follows the reference's definitions:
  * ``build_inv_dsq`` / ``inv_dsq``: js/crystal.js:326-377 (reciprocal metric as
    six coefficients, 1/d^2 as a quadratic form evaluated in the same order);
  * ``orth_matrix``: js/symmetry_utils.js:33-45 (fractional -> Cartesian, a along
    x, b in the xy plane; the reference rounds it to float32);
  * ``reduced_cell``: js/symmetry_utils.js:119-207 (pairwise Gauss reduction plus
    face-diagonal search; the reduced basis makes independent rounding of a
    fractional separation the nearest image out to ``safe_radius``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence

import numpy as np

DEG2RAD = math.pi / 180.0


def _cell(cell: Dict[str, float]):
    a = float(cell['a'])
    b = float(cell.get('b') or a) if (cell.get('b') or 0) > 0 else a
    c = float(cell.get('c') or a) if (cell.get('c') or 0) > 0 else a
    al = float(cell.get('alpha', 90.0) if cell.get('alpha') is not None else 90.0)
    be = float(cell.get('beta', 90.0) if cell.get('beta') is not None else 90.0)
    ga = float(cell.get('gamma', 90.0) if cell.get('gamma') is not None else 90.0)
    return a, b, c, al, be, ga


def build_inv_dsq(cell: Dict[str, float]) -> Optional[Dict[str, float]]:
    """Coefficients of 1/d^2 = h^2 aa + k^2 bb + l^2 cc + hk ab + kl bc + hl ac, or None."""
    a, b, c, al, be, ga = _cell(cell)
    if not (a > 0 and b > 0 and c > 0):
        return None
    al, be, ga = al * DEG2RAD, be * DEG2RAD, ga * DEG2RAD
    cosA, cosB, cosG = math.cos(al), math.cos(be), math.cos(ga)
    sinA, sinB, sinG = math.sin(al), math.sin(be), math.sin(ga)
    vf = 1 - cosA * cosA - cosB * cosB - cosG * cosG + 2 * cosA * cosB * cosG
    if vf <= 1e-9 or abs(sinA) < 1e-9 or abs(sinB) < 1e-9 or abs(sinG) < 1e-9:
        return None
    V = a * b * c * math.sqrt(vf)
    a_s = b * c * sinA / V
    b_s = a * c * sinB / V
    c_s = a * b * sinG / V
    cosA_s = (cosB * cosG - cosA) / (sinB * sinG)
    cosB_s = (cosA * cosG - cosB) / (sinA * sinG)
    cosG_s = (cosA * cosB - cosG) / (sinA * sinB)
    return {'aa': a_s * a_s, 'bb': b_s * b_s, 'cc': c_s * c_s,
            'ab': 2 * a_s * b_s * cosG_s, 'bc': 2 * b_s * c_s * cosA_s, 'ac': 2 * a_s * c_s * cosB_s}


def inv_dsq(f: Dict[str, float], h, k, l):
    """1/d^2, evaluated term by term left to right like the reference (works on arrays)."""
    return h * h * f['aa'] + k * k * f['bb'] + l * l * f['cc'] + h * k * f['ab'] + k * l * f['bc'] + h * l * f['ac']


def cell_volume(cell: Dict[str, float]) -> float:
    a, b, c, al, be, ga = _cell(cell)
    ca, cb, cg = (math.cos(v * DEG2RAD) for v in (al, be, ga))
    disc = 1 - ca * ca - cb * cb - cg * cg + 2 * ca * cb * cg
    return a * b * c * math.sqrt(disc) if disc > 0 else float('nan')


def orth_matrix(cell: Dict[str, float]) -> np.ndarray:
    """Fractional -> Cartesian (row-major 3x3), float32 like the reference."""
    a, b, c, al, be, ga = _cell(cell)
    al, be, ga = al * DEG2RAD, be * DEG2RAD, ga * DEG2RAD
    cosA, cosB, cosG, sinG = math.cos(al), math.cos(be), math.cos(ga), math.sin(ga)
    V = cell_volume(cell)
    return np.array([a, b * cosG, c * cosB,
                     0.0, b * sinG, c * (cosA - cosB * cosG) / sinG,
                     0.0, 0.0, V / (a * b * sinG)], dtype=np.float32)


def _widths(o: Sequence[float]) -> List[float]:
    a = np.array([o[0], o[3], o[6]], dtype=np.float64)
    b = np.array([o[1], o[4], o[7]], dtype=np.float64)
    c = np.array([o[2], o[5], o[8]], dtype=np.float64)
    vol = abs(float(np.dot(a, np.cross(b, c))))
    return [vol / float(np.linalg.norm(np.cross(b, c))), vol / float(np.linalg.norm(np.cross(c, a))),
            vol / float(np.linalg.norm(np.cross(a, b)))]


@dataclass
class ReducedCell:
    orth: np.ndarray      # fractional(reduced) -> Cartesian, row-major, float64
    xform: np.ndarray     # fractional(original) -> fractional(reduced), integer-valued, row-major
    safe_radius: float
    widths: List[float]
    changed: bool
    M: List[int]


def reduced_cell(cell: Dict[str, float]) -> ReducedCell:
    orth = orth_matrix(cell).astype(np.float64)
    v = [[orth[0], orth[3], orth[6]], [orth[1], orth[4], orth[7]], [orth[2], orth[5], orth[8]]]
    M = [[1, 0, 0], [0, 1, 0], [0, 0, 1]]

    def dot(p, q):
        return p[0] * q[0] + p[1] * q[1] + p[2] * q[2]

    def nrm(p):
        return dot(p, p)

    def sort_by_length():
        nonlocal v, M
        order = sorted(range(3), key=lambda i: nrm(v[i]))
        v = [v[i] for i in order]
        M = [M[i] for i in order]

    for _ in range(64):
        moved = False
        sort_by_length()
        for i in range(3):
            for j in range(3):
                if i == j:
                    continue
                nj = nrm(v[j])
                if not nj > 1e-12:
                    continue
                mu = math.floor(dot(v[i], v[j]) / nj + 0.5)  # JS Math.round
                if mu != 0:
                    v[i] = [v[i][k] - mu * v[j][k] for k in range(3)]
                    M[i] = [M[i][k] - mu * M[j][k] for k in range(3)]
                    moved = True
        sort_by_length()
        best, bestN = None, nrm(v[2])
        for c1 in (-1, 0, 1):
            for c2 in (-1, 0, 1):
                if not c1 and not c2:
                    continue
                t = [v[2][k] + c1 * v[0][k] + c2 * v[1][k] for k in range(3)]
                n = nrm(t)
                if n < bestN - 1e-9:
                    bestN, best = n, (c1, c2)
        if best:
            v[2] = [v[2][k] + best[0] * v[0][k] + best[1] * v[1][k] for k in range(3)]
            M[2] = [M[2][k] + best[0] * M[0][k] + best[1] * M[1][k] for k in range(3)]
            moved = True
        if not moved:
            break
    Mf = [M[0][0], M[0][1], M[0][2], M[1][0], M[1][1], M[1][2], M[2][0], M[2][1], M[2][2]]
    changed = Mf != [1, 0, 0, 0, 1, 0, 0, 0, 1]
    orthR = np.zeros(9)
    for r in range(3):
        for c in range(3):
            orthR[r * 3 + c] = sum(orth[r * 3 + k] * Mf[c * 3 + k] for k in range(3))
    Mi = np.linalg.inv(np.array(Mf, dtype=np.float64).reshape(3, 3))
    Minv = np.rint(Mi).astype(np.int64).reshape(-1)
    xform = np.array([Minv[0], Minv[3], Minv[6], Minv[1], Minv[4], Minv[7], Minv[2], Minv[5], Minv[8]],
                     dtype=np.float64)
    widths = _widths(orthR)
    return ReducedCell(orthR, xform, min(widths) / 2, widths, changed, Mf)


def inverse3(m: Sequence[float]) -> np.ndarray:
    """Inverse of a row-major 3x3 by the adjugate (swarm_wyckoff.js:1428-1436)."""
    c00 = m[4] * m[8] - m[5] * m[7]
    c01 = m[5] * m[6] - m[3] * m[8]
    c02 = m[3] * m[7] - m[4] * m[6]
    det = m[0] * c00 + m[1] * c01 + m[2] * c02
    inv = [c00, m[2] * m[7] - m[1] * m[8], m[1] * m[5] - m[2] * m[4],
           c01, m[0] * m[8] - m[2] * m[6], m[2] * m[3] - m[0] * m[5],
           c02, m[1] * m[6] - m[0] * m[7], m[0] * m[4] - m[1] * m[3]]
    return np.array([v / det for v in inv], dtype=np.float64)
