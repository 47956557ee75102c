"""Space-group operators and Wyckoff positions for the trial-evaluation path.

The reference reads its operators and Wyckoff tables from a cctbx-generated
database (``sg/all.json``; consumed by ``js/rietveld_core.js:139-180`` and
``js/wyckoff_assign.js:756-944``).  That database is not shipped here.  This
module builds the same objects from first principles instead:

* operators from a Hall symbol (Hall 1981, Acta Cryst. A37, 517; the notation
  of International Tables Vol. B, A1.4.2), closed into the full group with the
  lattice centring folded in, as the database's ``sym_ops`` are;
* Wyckoff positions from the International Tables coordinate triplet of each
  position.  The projector of a position is the average of its site-symmetry
  operators (the "special operator" the database stores as ``P_num/P_den``,
  ``T_num/T_den``), its coset operators are the first operator mapping a
  generic point of the position onto each image (``coset_ops``), and its number
  of free parameters is the rank of the projector (``n_free``).

Translations are held as integers in units of 1/24, so every operator is exact.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from fractions import Fraction
from typing import Dict, List, Sequence, Tuple

TDEN = 24  # translation unit: 1/24 of a cell edge

Mat = Tuple[int, ...]      # 9 ints, row-major
Vec = Tuple[int, int, int]  # translation numerators over TDEN


def _mul(a: Mat, b: Mat) -> Mat:
    return tuple(sum(a[3 * i + k] * b[3 * k + j] for k in range(3)) for i in range(3) for j in range(3))


def _mv(a: Mat, v: Sequence[int]) -> Tuple[int, int, int]:
    return tuple(a[3 * i] * v[0] + a[3 * i + 1] * v[1] + a[3 * i + 2] * v[2] for i in range(3))


IDENT: Mat = (1, 0, 0, 0, 1, 0, 0, 0, 1)
INV: Mat = (-1, 0, 0, 0, -1, 0, 0, 0, -1)

# Rotation matrices of the Hall notation, by principal axis and order.
_ROT = {
    'z': {1: IDENT,
          2: (-1, 0, 0, 0, -1, 0, 0, 0, 1),
          3: (0, -1, 0, 1, -1, 0, 0, 0, 1),
          4: (0, -1, 0, 1, 0, 0, 0, 0, 1),
          6: (1, -1, 0, 1, 0, 0, 0, 0, 1)},
    'x': {1: IDENT,
          2: (1, 0, 0, 0, -1, 0, 0, 0, -1),
          3: (1, 0, 0, 0, 0, -1, 0, 1, -1),
          4: (1, 0, 0, 0, 0, -1, 0, 1, 0),
          6: (1, 0, 0, 0, 1, -1, 0, 1, 0)},
    'y': {1: IDENT,
          2: (-1, 0, 0, 0, 1, 0, 0, 0, -1),
          3: (-1, 0, 1, 0, 1, 0, -1, 0, 0),
          4: (0, 0, 1, 0, 1, 0, -1, 0, 0),
          6: (0, 0, 1, 0, 1, 0, -1, 0, 1)},
}
# Two-fold axes along face diagonals, relative to the preceding principal axis.
_DIAG = {
    ("z", "'"): (0, -1, 0, -1, 0, 0, 0, 0, -1),
    ("z", '"'): (0, 1, 0, 1, 0, 0, 0, 0, -1),
    ("x", "'"): (-1, 0, 0, 0, 0, -1, 0, -1, 0),
    ("x", '"'): (-1, 0, 0, 0, 0, 1, 0, 1, 0),
    ("y", "'"): (0, 0, -1, 0, -1, 0, -1, 0, 0),
    ("y", '"'): (0, 0, 1, 0, -1, 0, 1, 0, 0),
}
_BODY3: Mat = (0, 0, 1, 1, 0, 0, 0, 1, 0)

_LATTICE = {
    'P': [], 'A': [(0, 12, 12)], 'B': [(12, 0, 12)], 'C': [(12, 12, 0)], 'I': [(12, 12, 12)],
    'R': [(16, 8, 8), (8, 16, 16)], 'S': [(8, 8, 16), (16, 16, 8)], 'T': [(8, 16, 8), (16, 8, 16)],
    'F': [(0, 12, 12), (12, 0, 12), (12, 12, 0)],
}
_TSYM = {'a': (12, 0, 0), 'b': (0, 12, 0), 'c': (0, 0, 12), 'n': (12, 12, 12),
         'u': (6, 0, 0), 'v': (0, 6, 0), 'w': (0, 0, 6), 'd': (6, 6, 6)}


@dataclass(frozen=True)
class SymOp:
    """One operator x' = R x + t, t in units of 1/24."""
    r: Mat
    t: Vec

    @property
    def t_frac(self) -> Tuple[float, float, float]:
        return tuple(v / TDEN for v in self.t)

    def compose(self, other: 'SymOp') -> 'SymOp':
        rt = _mv(self.r, other.t)
        return SymOp(_mul(self.r, other.r), tuple((rt[i] + self.t[i]) % TDEN for i in range(3)))


def _norm_t(t) -> Vec:
    return tuple(int(v) % TDEN for v in t)


def parse_hall(symbol: str) -> List[SymOp]:
    """Generators of a Hall symbol (lattice translations and inversion included)."""
    s = symbol.strip()
    shift = (0, 0, 0)
    if '(' in s:
        s, rest = s.split('(', 1)
        nums = rest.rstrip(')').split()
        shift = tuple(2 * int(v) for v in nums)  # twelfths -> 24ths
        s = s.strip()
    toks = s.split()
    lat = toks[0]
    centro = lat.startswith('-')
    lat = lat.lstrip('-').upper()
    if lat not in _LATTICE:
        raise ValueError(f'unknown lattice symbol in Hall symbol {symbol!r}')
    gens: List[SymOp] = [SymOp(IDENT, (0, 0, 0))]
    for c in _LATTICE[lat]:
        gens.append(SymOp(IDENT, c))
    if centro:
        gens.append(SymOp(INV, (0, 0, 0)))
    prev_n, prev_axis = None, None
    for idx, tok in enumerate(toks[1:]):
        improper = tok.startswith('-')
        body = tok.lstrip('-')
        n = int(body[0])
        rest = body[1:]
        screw = 0
        if rest and rest[0].isdigit():
            screw = int(rest[0])
            rest = rest[1:]
        axis = None
        if rest and rest[0] in "xyz'\"*":
            axis = rest[0]
            rest = rest[1:]
        if axis is None:
            if idx == 0:
                axis = 'z'
            elif idx == 1 and n == 2:
                axis = 'x' if prev_n in (2, 4) else "'"
            elif idx == 2 and n == 3:
                axis = '*'
            else:
                axis = 'z'
        if axis in ("'", '"'):
            r = _DIAG[(prev_axis or 'z', axis)]
            principal = prev_axis or 'z'
        elif axis == '*':
            r = _BODY3 if n == 3 else IDENT
            principal = '*'
        else:
            r = _ROT[axis][n]
            principal = axis
        if improper:
            r = tuple(-v for v in r)
        t = [0, 0, 0]
        for ch in rest:
            tv = _TSYM[ch]
            t = [t[i] + tv[i] for i in range(3)]
        if screw:
            step = TDEN * screw // n
            ax = {'x': 0, 'y': 1, 'z': 2}.get(principal)
            if ax is None:
                raise ValueError(f'screw on a non-principal axis in {symbol!r}')
            t[ax] += step
        gens.append(SymOp(r, _norm_t(t)))
        if axis in 'xyz':
            prev_axis = axis
        prev_n = n
    if any(shift):
        # change of origin by v: (R, t) -> (R, t + (R - I) v) with v the shift
        out = []
        for g in gens:
            rv = _mv(g.r, shift)
            out.append(SymOp(g.r, _norm_t(tuple(g.t[i] + rv[i] - shift[i] for i in range(3)))))
        gens = out
    return gens


def close_group(gens: Sequence[SymOp], limit: int = 4096) -> List[SymOp]:
    """Closure of a generator set, identity first, then in discovery order."""
    ident = SymOp(IDENT, (0, 0, 0))
    ops = [ident]
    seen = {ident}
    frontier = [ident]
    gens = [g for g in gens]
    while frontier:
        nxt = []
        for a in frontier:
            for g in gens:
                for c in (a.compose(g), g.compose(a)):
                    if c not in seen:
                        seen.add(c)
                        ops.append(c)
                        nxt.append(c)
                        if len(ops) > limit:
                            raise ValueError('group closure exceeded the operator limit')
        frontier = nxt
    return ops


# ---------------------------------------------------------------------------
# Wyckoff positions (International Tables, standard settings), highest
# multiplicity first as the database lists them.
# ---------------------------------------------------------------------------
_WYCKOFF: Dict[str, List[Tuple[str, int, str]]] = {
    'P 1': [('a', 1, 'x,y,z')],
    '-P 1': [('i', 2, 'x,y,z'), ('h', 1, '1/2,1/2,1/2'), ('g', 1, '0,1/2,1/2'), ('f', 1, '1/2,0,1/2'),
             ('e', 1, '1/2,1/2,0'), ('d', 1, '1/2,0,0'), ('c', 1, '0,1/2,0'), ('b', 1, '0,0,1/2'),
             ('a', 1, '0,0,0')],
    '-P 2ybc': [('e', 4, 'x,y,z'), ('d', 2, '1/2,0,1/2'), ('c', 2, '0,0,1/2'), ('b', 2, '1/2,0,0'),
                ('a', 2, '0,0,0')],
    '-C 2yc': [('f', 8, 'x,y,z'), ('e', 4, '0,y,1/4'), ('d', 4, '1/4,1/4,1/2'), ('c', 4, '1/4,1/4,0'),
               ('b', 4, '0,1/2,0'), ('a', 4, '0,0,0')],
    '-C 2y': [('j', 8, 'x,y,z'), ('i', 4, 'x,0,z'), ('h', 4, '0,y,1/2'), ('g', 4, '0,y,0'),
              ('f', 4, '1/4,1/4,1/2'), ('e', 4, '1/4,1/4,0'), ('d', 2, '0,1/2,1/2'), ('c', 2, '0,0,1/2'),
              ('b', 2, '0,1/2,0'), ('a', 2, '0,0,0')],
    '-P 2ac 2n': [('d', 8, 'x,y,z'), ('c', 4, 'x,1/4,z'), ('b', 4, '0,0,1/2'), ('a', 4, '0,0,0')],
    '-P 6c': [('i', 12, 'x,y,z'), ('h', 6, 'x,y,1/4'), ('g', 6, '1/2,0,0'), ('f', 4, '1/3,2/3,z'),
              ('e', 4, '0,0,z'), ('d', 2, '2/3,1/3,1/4'), ('c', 2, '1/3,2/3,1/4'), ('b', 2, '0,0,0'),
              ('a', 2, '0,0,1/4')],
    '-F 4 2 3': [('l', 192, 'x,y,z'), ('k', 96, 'x,x,z'), ('j', 96, '0,y,z'), ('i', 48, '1/2,y,y'),
                 ('h', 48, '0,y,y'), ('g', 48, 'x,1/4,1/4'), ('f', 32, 'x,x,x'), ('e', 24, 'x,0,0'),
                 ('d', 24, '0,1/4,1/4'), ('c', 8, '1/4,1/4,1/4'), ('b', 4, '1/2,1/2,1/2'),
                 ('a', 4, '0,0,0')],
    '-P 4 2 3': [('n', 48, 'x,y,z'), ('m', 24, 'x,x,z'), ('l', 24, '1/2,y,z'), ('k', 24, '0,y,z'),
                 ('j', 12, '1/2,y,y'), ('i', 12, '0,y,y'), ('h', 12, 'x,1/2,0'), ('g', 8, 'x,x,x'),
                 ('f', 6, 'x,1/2,1/2'), ('e', 6, 'x,0,0'), ('d', 3, '1/2,0,0'), ('c', 3, '0,1/2,1/2'),
                 ('b', 1, '1/2,1/2,1/2'), ('a', 1, '0,0,0')],
    '-P 4 2': [('u', 16, 'x,y,z'), ('t', 8, 'x,1/2,z'), ('s', 8, 'x,0,z'), ('r', 8, 'x,x,z'), ('q', 8, 'x,y,1/2'),
               ('p', 8, 'x,y,0'), ('o', 4, 'x,1/2,1/2'), ('n', 4, 'x,1/2,0'), ('m', 4, 'x,0,1/2'),
               ('l', 4, 'x,0,0'), ('k', 4, 'x,x,1/2'), ('j', 4, 'x,x,0'), ('i', 4, '0,1/2,z'), ('h', 2, '1/2,1/2,z'),
               ('g', 2, '0,0,z'), ('f', 2, '0,1/2,0'), ('e', 2, '0,1/2,1/2'), ('d', 1, '1/2,1/2,1/2'),
               ('c', 1, '1/2,1/2,0'), ('b', 1, '0,0,1/2'), ('a', 1, '0,0,0')],
    '-R 3 2"': [('i', 36, 'x,y,z'), ('h', 18, 'x,-x,z'), ('g', 18, 'x,0,1/2'), ('f', 18, 'x,0,0'),
                ('e', 9, '1/2,0,0'), ('d', 9, '1/2,0,1/2'), ('c', 6, '0,0,z'), ('b', 3, '0,0,1/2'),
                ('a', 3, '0,0,0')],
}

# Space groups this module builds: number -> (symbol, Hall symbol, crystal system).
SPACE_GROUPS: Dict[int, Tuple[str, str, str]] = {
    1: ('P1', 'P 1', 'triclinic'),
    2: ('P-1', '-P 1', 'triclinic'),
    12: ('C2/m', '-C 2y', 'monoclinic'),
    14: ('P2_1/c', '-P 2ybc', 'monoclinic'),
    15: ('C2/c', '-C 2yc', 'monoclinic'),
    62: ('Pnma', '-P 2ac 2n', 'orthorhombic'),
    123: ('P4/mmm', '-P 4 2', 'tetragonal'),
    166: ('R-3m:H', '-R 3 2"', 'trigonal'),
    176: ('P6_3/m', '-P 6c', 'hexagonal'),
    221: ('Pm-3m', '-P 4 2 3', 'cubic'),
    225: ('Fm-3m', '-F 4 2 3', 'cubic'),
}

_GENERIC = (Fraction(7, 61), Fraction(11, 59), Fraction(17, 53))


def _parse_triplet(trip: str) -> List[Tuple[Tuple[Fraction, Fraction, Fraction], Fraction]]:
    """'x,1/4,z' -> per component (coefficients of x,y,z; constant)."""
    out = []
    for comp in trip.replace(' ', '').split(','):
        coef = [Fraction(0)] * 3
        const = Fraction(0)
        i = 0
        sign = 1
        term = ''
        comp = comp + '+'
        while i < len(comp):
            ch = comp[i]
            if ch in '+-' and term:
                if term[-1] in 'xyz':
                    num = term[:-1]
                    f = Fraction(1) if num in ('', '+') else Fraction(num.rstrip('*'))
                    coef['xyz'.index(term[-1])] += sign * f
                else:
                    const += sign * Fraction(term)
                term = ''
                sign = 1 if ch == '+' else -1
            elif ch in '+-':
                sign = 1 if ch == '+' else -1
            else:
                term += ch
            i += 1
        out.append((tuple(coef), const))
    return out


def _frac_mod1(v: Fraction) -> Fraction:
    return v - (v.numerator // v.denominator)


@dataclass
class WyckoffPosition:
    letter: str
    multiplicity: int
    triplet: str
    P: Tuple[Fraction, ...]        # 9 entries, the special operator's linear part
    T: Tuple[Fraction, Fraction, Fraction]
    n_free: int
    coset_ops: List[int]
    site_symmetry_order: int

    @property
    def P_float(self) -> List[float]:
        return [float(v) for v in self.P]

    @property
    def T_float(self) -> List[float]:
        return [float(v) for v in self.T]

    def project(self, x: float, y: float, z: float) -> Tuple[float, float, float]:
        P, T = self.P_float, self.T_float
        return tuple(P[3 * i] * x + P[3 * i + 1] * y + P[3 * i + 2] * z + T[i] for i in range(3))


def _rank(m: List[List[Fraction]]) -> int:
    a = [row[:] for row in m]
    rank = 0
    rows, cols = len(a), len(a[0])
    for c in range(cols):
        piv = next((r for r in range(rank, rows) if a[r][c] != 0), None)
        if piv is None:
            continue
        a[rank], a[piv] = a[piv], a[rank]
        for r in range(rows):
            if r != rank and a[r][c] != 0:
                f = a[r][c] / a[rank][c]
                a[r] = [a[r][k] - f * a[rank][k] for k in range(cols)]
        rank += 1
    return rank


def build_wyckoff(ops: Sequence[SymOp], letter: str, mult: int, triplet: str) -> WyckoffPosition:
    comps = _parse_triplet(triplet)
    # the generic point is kept unreduced so T is the constant of the triplet itself
    p0 = tuple(sum(c[0][k] * _GENERIC[k] for k in range(3)) + c[1] for c in comps)
    stab = []
    for op in ops:
        q = [sum(op.r[3 * i + k] * p0[k] for k in range(3)) + Fraction(op.t[i], TDEN) for i in range(3)]
        d = [p0[i] - q[i] for i in range(3)]
        if all(v.denominator == 1 for v in d):
            stab.append((op, d))
    n = len(stab)
    P = [Fraction(0)] * 9
    T = [Fraction(0)] * 3
    for op, d in stab:
        for k in range(9):
            P[k] += Fraction(op.r[k], n)
        for i in range(3):
            T[i] += (Fraction(op.t[i], TDEN) + d[i]) / n
    # cosets: first operator per distinct image of the generic point
    images: List[Tuple[Fraction, ...]] = []
    cos: List[int] = []
    for idx, op in enumerate(ops):
        q = tuple(_frac_mod1(sum(op.r[3 * i + k] * p0[k] for k in range(3)) + Fraction(op.t[i], TDEN))
                  for i in range(3))
        if q not in images:
            images.append(q)
            cos.append(idx)
    if len(cos) != mult or len(ops) // n != mult:
        raise ValueError(f'Wyckoff {mult}{letter} ({triplet}): orbit of {len(cos)} images, '
                         f'site symmetry of order {n} in a group of {len(ops)}')
    rank = _rank([[P[3 * i + k] for k in range(3)] for i in range(3)])
    return WyckoffPosition(letter, mult, triplet, tuple(P), tuple(T), rank, cos, n)


@dataclass
class SpaceGroup:
    number: int
    symbol: str
    hall: str
    system: str
    ops: List[SymOp]
    wyckoff: List[WyckoffPosition] = field(default_factory=list)
    unique_axis: str = 'b'

    @property
    def order(self) -> int:
        return len(self.ops)

    def position(self, label: str) -> WyckoffPosition:
        """'4c' or 'c' -> the Wyckoff position."""
        letter = label.strip()[-1]
        for w in self.wyckoff:
            if w.letter == letter:
                return w
        raise KeyError(f'{self.symbol} has no Wyckoff position {label!r}')

    def op_dicts(self) -> List[dict]:
        """Operators in the database's shape: r (9 ints) and t (floats)."""
        return [{'r': list(o.r), 't': list(o.t_frac), 't_num': list(o.t), 't_den': TDEN} for o in self.ops]


_CACHE: Dict[int, SpaceGroup] = {}


def space_group(number: int) -> SpaceGroup:
    if number in _CACHE:
        return _CACHE[number]
    if number not in SPACE_GROUPS:
        raise KeyError(f'space group {number} is not tabulated here; available: {sorted(SPACE_GROUPS)}')
    sym, hall, system = SPACE_GROUPS[number]
    ops = close_group(parse_hall(hall))
    g = SpaceGroup(number, sym, hall, system, ops)
    g.wyckoff = [build_wyckoff(ops, l, m, t) for (l, m, t) in _WYCKOFF[hall]]
    _CACHE[number] = g
    return g


def group_from_hall(hall: str) -> List[SymOp]:
    return close_group(parse_hall(hall))


# ---------------------------------------------------------------------------
# Operator algebra of the reference (js/rietveld_core.js:127-201,
# js/swarm_wyckoff.js:301-312, js/wyckoff_assign.js:772-781)
# ---------------------------------------------------------------------------

def centring_vectors(ops: Sequence[SymOp]) -> List[Tuple[float, float, float]]:
    """Pure translations of the group (wyckoff_assign.js:772-781)."""
    return [o.t_frac for o in ops if o.r == IDENT and any(o.t)]


def cosets(ops: Sequence[SymOp]) -> Tuple[List[SymOp], int]:
    """Coset representatives modulo centring, and the centring count (rietveld_core.js:164-180)."""
    cen = [o.t for o in ops if o.r == IDENT]
    reps: List[SymOp] = []
    for o in ops:
        dup = False
        for q in reps:
            if q.r != o.r:
                continue
            for c in cen:
                if all((o.t[i] - q.t[i] - c[i]) % TDEN == 0 for i in range(3)):
                    dup = True
                    break
            if dup:
                break
        if not dup:
            reps.append(o)
    return reps, len(cen)


def laue_rotations(ops: Sequence[SymOp]) -> List[Mat]:
    """Rotation parts with Friedel's law added, deduplicated (rietveld_core.js:182-188)."""
    seen = {}
    for o in ops:
        for r in (o.r, tuple(-v for v in o.r)):
            if r not in seen:
                seen[r] = r
    return list(seen.values())


def has_inversion_at_origin(ops: Sequence[SymOp]) -> bool:
    """(-I | 0) in the group (swarm_wyckoff.js:301-312)."""
    return any(o.r == INV and not any(o.t) for o in ops)


__all__ = ['SymOp', 'SpaceGroup', 'WyckoffPosition', 'space_group', 'group_from_hall', 'parse_hall',
           'close_group', 'build_wyckoff', 'cosets', 'laue_rotations', 'has_inversion_at_origin',
           'centring_vectors', 'SPACE_GROUPS', 'TDEN', 'IDENT', 'INV']
