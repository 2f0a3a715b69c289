"""Build libdesv.so (all CUDA kernels + the C ABI) in-tree for sm_100a.

    python dense-evolution_b200/build.py [--verbose] [--ptxas-info]

Objects go to dense-evolution_b200/_build/, the library to
dense-evolution_b200/dense_evolution/_lib/libdesv.so, next to the Python
package that loads it.  nvcc cross-compiles without a GPU.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, 'csrc')
BUILD = os.path.join(PKG, '_build')
LIBDIR = os.path.join(PKG, 'dense_evolution', '_lib')
LIB = os.path.join(LIBDIR, 'libdesv.so')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
FLAGS = ['-O3', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC', '-Xcompiler', '-O2',
         '--expt-relaxed-constexpr', '-I', os.path.join(ROOT, 'include'), '-I', CSRC]


def nvcc() -> str:
    for c in (os.environ.get('NVCC'), '/usr/local/cuda/bin/nvcc', shutil.which('nvcc')):
        if c and os.path.exists(c):
            return c
    raise RuntimeError('nvcc not found')


def _needs(obj: str, deps) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, '*.cu')))
    headers = glob.glob(os.path.join(CSRC, '*.cuh')) + glob.glob(os.path.join(ROOT, 'include', '*.h'))
    cc = nvcc()
    extra = ['-Xptxas', '-v'] if ptxas_info else []

    def compile_one(src):
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + '.o')
        if not force and not ptxas_info and not _needs(obj, [src, *headers, __file__]):
            return obj, ''
        cmd = [cc, *ARCH, *FLAGS, *extra, '-c', src, '-o', obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f'nvcc failed for {src}:\n{r.stdout}\n{r.stderr}')
        return obj, r.stderr

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(compile_one, srcs))
    objs = [o for o, _ in results]
    if verbose or ptxas_info:
        for _, log in results:
            if log:
                print(log)
    if force or ptxas_info or _needs(LIB, objs):
        cmd = [cc, *ARCH, '-shared', '-o', LIB, *objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f'link failed:\n{r.stdout}\n{r.stderr}')
    return LIB


if __name__ == '__main__':
    ap = argparse.ArgumentParser()
    ap.add_argument('--verbose', action='store_true')
    ap.add_argument('--ptxas-info', action='store_true')
    ap.add_argument('--force', action='store_true')
    a = ap.parse_args()
    print(build(a.verbose, a.ptxas_info, a.force))
    sys.exit(0)
