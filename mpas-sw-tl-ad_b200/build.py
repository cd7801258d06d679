"""Build the engine library ``libmpsw.so`` in place (next to this file).

Every translation unit targets sm_100a only.  The FP64 stencils (``csrc/mpsw_f64.cu``) and the
host set-up are compiled without floating-point contraction so the FP64 path performs the
reference's roundings one operation at a time; the FP32-stencil unit allows FMA.  The CUDA
runtime is linked statically so the library does not depend on the runtime bundled with any
Python package.

Usage: ``python build.py`` (or ``import build; build.build()``).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
INCLUDE = os.path.join(os.path.dirname(HERE), 'include')
OUT_DIR = os.path.join(HERE, '_build')
LIB = os.path.join(HERE, 'libmpsw.so')

ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
NVCC_COMMON = ['-std=c++17', '-O3', '-lineinfo', '-Xcompiler', '-fPIC', '-Xcompiler',
               '-ffp-contract=off', '-I' + CSRC, '-I' + INCLUDE] + ARCH

UNITS = [
    ('mpsw_f64.cu', ['--fmad=false']),
    ('mpsw_f32.cu', ['--fmad=true']),
    ('mpsw_engine.cu', ['--fmad=false']),
    ('mpsw_window.cu', ['--fmad=false']),
    ('mpsw_noalloc.cu', ['--fmad=false']),
    ('mpsw_ic.cu', ['--fmad=false']),
    ('mpsw_testcases.cu', ['--fmad=false']),
    ('mpsw_setup.cpp', ['--fmad=false', '-x', 'cu']),
    ('mpsw_tiles.cpp', ['--fmad=false', '-x', 'cu']),
]
HEADERS = ['mpsw_internal.h', 'mpsw_kernels.cuh', 'mpsw_launch.h', 'mpsw_launch.cuh', 'mpsw_members.cuh',
           'mpsw_fused.cuh', 'mpsw_setup.h', 'mpsw_tiles.h', 'mpsw_engine.h']


def _nvcc():
    exe = shutil.which('nvcc') or '/usr/local/cuda/bin/nvcc'
    if not os.path.exists(exe):
        raise RuntimeError('nvcc not found')
    return exe


def _newest_dep():
    paths = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, 'mpsw.h'),
                                                         os.path.abspath(__file__)]
    return max(os.path.getmtime(p) for p in paths if os.path.exists(p))


def build(verbose: bool = False, force: bool = False) -> str:
    """Compile and link ``libmpsw.so``; returns its path.  Incremental on file times."""
    os.makedirs(OUT_DIR, exist_ok=True)
    nvcc = _nvcc()
    dep_time = _newest_dep()
    objs = []
    for src, flags in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(OUT_DIR, os.path.splitext(src)[0] + '.o')
        objs.append(o)
        if (not force and os.path.exists(o) and os.path.getmtime(o) >= os.path.getmtime(s)
                and os.path.getmtime(o) >= dep_time):
            continue
        cmd = [nvcc] + NVCC_COMMON + flags + ['-c', s, '-o', o]
        if verbose:
            print(' '.join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        tmp = LIB + '.tmp'
        cmd = [nvcc] + ARCH + ['-shared', '-cudart', 'static', '-o', tmp] + objs + ['-lpthread', '-ldl', '-lrt']
        if verbose:
            print(' '.join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        os.replace(tmp, LIB)
    return LIB


if __name__ == '__main__':
    print(build(verbose=True, force='--force' in sys.argv))
