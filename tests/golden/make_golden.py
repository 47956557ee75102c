"""Generate the committed golden fixtures from the reference's own data files.

Run where the reference tree is available, giving its path:

    python tests/golden/make_golden.py <reference tree>

It reads, read-only:
  * sg/all.json (the cctbx-generated space-group database the reference ships):
    for every space group this package builds, the standard setting's Hall
    symbol, its operators, and each Wyckoff position's multiplicity, free
    parameter count, projector (P, T) and the orbit of a fixed generic point;
  * scatters/xray_wk1995_ions.json: the five-Gaussian coefficients of the few
    elements the tests and benchmarks use (Waasmaier & Kirfel, Acta Cryst. A51
    (1995) 416, as tabulated by cctbx);
  * test_files/cimetidine/cime.pdb: cimetidine's 17 non-hydrogen atoms and
    their bonds, the molecule of the learned-proposal workload.

Only derived, compact records are written (operator sets as integers over 24,
rational projectors, orbit coordinates); nothing else from the reference tree is
copied.  The fixtures let the tests pin this package's own operator and Wyckoff
construction against the reference's database without the database present.
"""
import json
import sys
from fractions import Fraction
from pathlib import Path

HERE = Path(__file__).resolve().parent
# number -> Hall symbol of the setting pinned (International Tables standard settings;
# monoclinic groups in unique axis b, cell choice 1)
GROUPS = {1: 'P 1', 2: '-P 1', 12: '-C 2y', 14: '-P 2ybc', 15: '-C 2yc', 62: '-P 2ac 2n', 123: '-P 4 2',
          166: '-R 3 2"', 176: '-P 6c', 221: '-P 4 2 3', 225: '-F 4 2 3'}
ELEMENTS = ['H', 'C', 'N', 'O', 'Na', 'S', 'Cl', 'Pb', 'Ti', 'Fe']
GENERIC = (0.1234, 0.3721, 0.5873)


def setting_by_hall(g, hall):
    for s in g['settings']:
        if s['hall'].strip() == hall:
            return s
    raise KeyError(hall)


def main(ref_root):
    ref = Path(ref_root)
    db = json.loads((ref / 'sg' / 'all.json').read_text())['space_groups']
    out = {}
    for n, hall in GROUPS.items():
        g = db[str(n)]
        s = setting_by_hall(g, hall)
        ops = []
        for o in s['sym_ops']:
            t = [int(Fraction(int(v), int(o['t_den'])) * 24) % 24 for v in o['t_num']]
            ops.append([int(v) for v in o['r']] + t)
        ops.sort()
        wy = []
        for w in s['wyckoff']:
            P = [str(Fraction(int(v), int(w['P_den']))) for v in w['P_num']]
            T = [str(Fraction(int(v), int(w['T_den']))) for v in w['T_num']]
            Pf = [float(Fraction(p)) for p in P]
            Tf = [float(Fraction(t)) for t in T]
            p = [sum(Pf[3 * i + k] * GENERIC[k] for k in range(3)) + Tf[i] for i in range(3)]
            orbit = []
            for oi in w['coset_ops']:
                o = s['sym_ops'][oi]
                r = o['r']
                t = [int(v) / int(o['t_den']) for v in o['t_num']]
                q = [sum(r[3 * i + k] * p[k] for k in range(3)) + t[i] for i in range(3)]
                orbit.append([round(v - __import__('math').floor(v), 9) % 1.0 for v in q])
            orbit.sort()
            wy.append({'letter': w['letter'], 'multiplicity': int(w['multiplicity']),
                       'n_free': int(w['n_free']), 'P': P, 'T': T, 'orbit': orbit})
        out[str(n)] = {'symbol': s['symbol'], 'hall': s['hall'], 'ops': ops, 'wyckoff': wy}
    (HERE / 'sg_fixture.json').write_text(json.dumps(out, separators=(',', ':')))

    xr = json.loads((ref / 'scatters' / 'xray_wk1995_ions.json').read_text())['table']
    ff = {}
    for e in ELEMENTS:
        rec = xr[e]
        ff[e] = {'Z': rec['Z'], 'a': rec['a'], 'b': rec['b'], 'c': rec['c']}
    text = json.dumps({'source': 'Waasmaier & Kirfel (1995), five-Gaussian f0, via the reference scattering table',
                       'table': ff}, indent=1)
    # the package reads the coefficients for its synthetic workloads (one copy, package data)
    ff_path = HERE.parent.parent / 'powder6_b200' / 'data' / 'xray_wk1995_subset.json'
    ff_path.write_text(text)
    # the config-5 molecule: cimetidine's non-hydrogen atoms (element, Cartesian A) and their bonds,
    # from the reference's test file test_files/cimetidine/cime.pdb (ATOM records and CONECT)
    atoms, serial_of, bonds = [], {}, set()
    for line in (ref / 'test_files' / 'cimetidine' / 'cime.pdb').read_text().splitlines():
        if line.startswith(('ATOM', 'HETATM')):
            el = line[76:78].strip() or line[12:16].strip()[:1]
            if el.upper() == 'H':
                continue
            serial_of[int(line[6:11])] = len(atoms)
            atoms.append({'element': el.capitalize(), 'xyz': [float(line[30:38]), float(line[38:46]),
                                                               float(line[46:54])]})
        elif line.startswith('CONECT'):
            nums = [int(v) for v in line[6:].split()[:5] if v.isdigit()]
            for other in nums[1:]:
                if nums[0] in serial_of and other in serial_of:
                    bonds.add(tuple(sorted((serial_of[nums[0]], serial_of[other]))))
    mol_path = HERE.parent.parent / 'powder6_b200' / 'data' / 'cimetidine_heavy.json'
    mol_path.write_text(json.dumps({'source': 'cimetidine, non-hydrogen atoms of the reference test file',
                                    'atoms': atoms, 'bonds': sorted(bonds)}, indent=1))
    print('wrote', HERE / 'sg_fixture.json', ff_path, mol_path)


if __name__ == '__main__':
    if len(sys.argv) != 2:
        sys.exit('usage: python tests/golden/make_golden.py <path of the reference tree>')
    main(sys.argv[1])
