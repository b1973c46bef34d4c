"""Builds the in-tree shared libraries of the GPU numeric phase for sm_100a.

    python -m sam_lib_b200.build        (or __graft_entry__.build())

Outputs (next to this file, git-ignored, shipped with the tree):
    libspr_b200.so      INTEGER*8 ABI (the default SPR_I8 build)
    libspr_b200_i4.so   INTEGER*4 ABI (BUILD_SPR_INTEGER8=OFF)
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
BUILD = os.path.join(HERE, '_build')
NVCC = os.environ.get('NVCC', 'nvcc')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
COMMON = ['-O3', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC', '-Xcompiler', '-O3', '-Xcompiler', '-ffp-contract=off']

ENGINE_SOURCES = ['engine.cu', 'plan.cpp', 'noalloc.cu', 'elements.cu']


def _run(cmd):
    print(' '.join(cmd), flush=True)
    subprocess.check_call(cmd)


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose_ptxas=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(('.h', '.cuh'))]
    objs = []
    for src in ENGINE_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + '.o')
        if _newer(o, [s] + headers + [__file__]):
            extra = ['-Xptxas', '-v'] if (verbose_ptxas and src.endswith('.cu')) else []
            _run([NVCC] + ARCH + COMMON + extra + ['-c', s, '-o', o])
        objs.append(o)
    outs = []
    for name, defs in (('libspr_b200.so', ['-DSPR_INT=int64_t']),
                       ('libspr_b200_i4.so', ['-DSPR_INT=int32_t'])):
        s = os.path.join(CSRC, 'abi.cpp')
        o = os.path.join(BUILD, name + '.abi.o')
        if _newer(o, [s] + headers + [__file__]):
            _run([NVCC] + ARCH + COMMON + defs + ['-c', s, '-o', o])
        so = os.path.join(HERE, name)
        if _newer(so, objs + [o]):
            _run([NVCC] + ARCH + ['-shared', '-cudart', 'static', '-o', so] + objs + [o])
        outs.append(so)
    return outs


if __name__ == '__main__':
    build(verbose_ptxas='-v' in sys.argv)
