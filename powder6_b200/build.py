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
    """Each source compiled to an object in parallel (objects in _build/),
    then linked into the shared library."""
    if not force and not needs_build():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    obj_dir = ROOT / '_build'
    obj_dir.mkdir(exist_ok=True)
    nvcc = nvcc_path()
    flags = [*ARCH, '-O3', '-lineinfo', '-std=c++17', '--use_fast_math', '-Xcompiler', '-fPIC',
             '-I', str(ROOT / 'include')]
    if verbose:
        flags.insert(0, '-Xptxas=-v')

    headers = [q for q in list(CSRC.glob('*.cuh')) + list(CSRC.glob('*.h')) + [ROOT / 'include' / 'p6cuda.h']
               if q.is_file()]
    newest_header = max((q.stat().st_mtime for q in headers), default=0.0)

    def compile_one(src: Path):
        obj = obj_dir / (src.stem + '.o')
        if (not force and not verbose and obj.exists() and obj.stat().st_mtime > src.stat().st_mtime
                and obj.stat().st_mtime > newest_header):
            return src, obj, subprocess.CompletedProcess([], 0, '', '')   # object up to date
        return src, obj, subprocess.run([nvcc, *flags, '-c', str(src), '-o', str(obj)], capture_output=True, text=True)

    srcs = sorted(sources(), key=lambda q: -q.stat().st_size)   # the largest first
    with ThreadPoolExecutor(max_workers=max(1, min(len(srcs), os.cpu_count() or 1))) as ex:
        results = list(ex.map(compile_one, srcs))
    for src, obj, res in results:
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError(f'nvcc failed on {src.name}')
        if verbose:
            sys.stderr.write(res.stderr)
    link = subprocess.run([nvcc, *ARCH, '-shared', '-o', str(LIB) + '.tmp', *[str(o) for _, o, _ in results]],
                          capture_output=True, text=True)
    if link.returncode != 0:
        sys.stderr.write(link.stdout + link.stderr)
        raise RuntimeError('nvcc failed linking libp6cuda.so')
    os.replace(str(LIB) + '.tmp', LIB)
    return LIB


if __name__ == '__main__':
    ap = argparse.ArgumentParser()
    ap.add_argument('--verbose', action='store_true')
    ap.add_argument('--force', action='store_true')
    a = ap.parse_args()
    print(build(verbose=a.verbose, force=a.force))
