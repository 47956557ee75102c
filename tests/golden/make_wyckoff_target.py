"""Writes tests/golden/wyckoff_target.json: the converged wR2 of the PbSO4-like
Pnma search (4096 replicas x 5000 generations, the reference's resolution and
penalty ramps) as the FP64 CPU port of the trial evaluation reaches it
(oracle.WyckoffCpuRunner: Metropolis per replica at fixed rung temperatures,
OpenMP over replicas).  The best cc at full resolution and the final penalty
weight, over every replica and every generation of the full-resolution tail
of the schedule, gives the converged wR2 = 1 - cc; the time-to-target of the
GPU searches is measured against 1.05 x that value, so the target does not
come from the system being timed.

    python tests/golden/make_wyckoff_target.py     (about two minutes on 8 cores)
"""
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402
from powder6_b200.swarm_wyckoff import schedule  # noqa: E402
from powder6_b200.workloads import wyckoff_problem  # noqa: E402

REPLICAS, GENERATIONS = 4096, 5000


def main():
    P = wyckoff_problem(seed=1)
    groups, pen = schedule(GENERATIONS, P.refl.n_groups)
    r = O.WyckoffCpuRunner(P, REPLICAS, seed=20261026)
    t0 = time.perf_counter()
    best = -np.inf
    for g in range(GENERATIONS):
        r.generation(int(groups[g]), float(pen[g]))
        if groups[g] == P.refl.n_groups and pen[g] == pen[-1]:
            st = r.st.reshape(REPLICAS, 8)
            best = max(best, float(np.max(st[:, 1])))
    dt = time.perf_counter() - t0
    wr2 = 1.0 - best
    out = {'workload': 'wyckoff-search Pnma PbSO4-like, wyckoff_problem(seed=1)', 'replicas': REPLICAS,
           'generations': GENERATIONS, 'converged_wr2': wr2, 'target_wr2': 1.05 * wr2,
           'seconds': round(dt, 1), 'threads': O.num_threads(),
           'source': 'FP64 CPU port of the trial evaluation, best full-resolution cc over the schedule tail'}
    (Path(__file__).parent / 'wyckoff_target.json').write_text(json.dumps(out, indent=1) + '\n')
    print(out)


if __name__ == '__main__':
    main()
