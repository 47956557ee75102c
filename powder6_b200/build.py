"""In-tree build of libp6cuda.so for sm_100a (nvcc, no JIT cache).

    python -m powder6_b200.build          # builds powder6_b200/libp6cuda.so
    python -m powder6_b200.build --verbose  # prints ptxas register / spill usage

The shared library is git-ignored and rebuilt from the sources here.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / 'csrc'
LIB = PKG / 'libp6cuda.so'
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']


def nvcc_path() -> str:
    for cand in (os.environ.get('NVCC'), shutil.which('nvcc'), '/usr/local/cuda/bin/nvcc'):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError('nvcc not found: set NVCC or install the CUDA toolkit')


def sources():
    return sorted(CSRC.glob('*.cu'))


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = list(CSRC.glob('*')) + [ROOT / 'include' / 'p6cuda.h']
    return any(p.stat().st_mtime > t for p in deps if p.is_file())


def build(verbose: bool = False, force: bool = False) -> Path:
    if not force and not needs_build():
        return LIB
    cmd = [nvcc_path(), *ARCH, '-O3', '-lineinfo', '-std=c++17', '--use_fast_math',
           '-Xcompiler', '-fPIC', '-shared', '-I', str(ROOT / 'include'),
           '-o', str(LIB) + '.tmp', *map(str, sources())]
    if verbose:
        cmd.insert(1, '-Xptxas=-v')
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError('nvcc failed building libp6cuda.so')
    if verbose:
        sys.stderr.write(res.stderr)
    os.replace(str(LIB) + '.tmp', LIB)
    return LIB


if __name__ == '__main__':
    ap = argparse.ArgumentParser()
    ap.add_argument('--verbose', action='store_true')
    ap.add_argument('--force', action='store_true')
    a = ap.parse_args()
    print(build(verbose=a.verbose, force=a.force))
