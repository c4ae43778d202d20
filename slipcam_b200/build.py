"""
Build the CUDA library libslipcam_b200.so in the package directory (sm_100a only).

usage: python -m slipcam_b200.build [--force]
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
LIB = os.path.join(HERE, 'libslipcam_b200.so')
SOURCES = ['capi.cu', 'diff.cu', 'multi.cu', 'stabilize.cu', 'warp.cu']
NVCC = os.environ.get('NVCC', '/usr/local/cuda/bin/nvcc')
FLAGS = ['-std=c++17', '-O3', '--expt-relaxed-constexpr', '-gencode', 'arch=compute_100a,code=sm_100a',
         '-lineinfo', '-Xcompiler', '-fPIC', '-Xcompiler', '-fvisibility=hidden', '-diag-suppress', '20014']
LINK = ['-gencode', 'arch=compute_100a,code=sm_100a', '-shared', '-cudart', 'static']


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(os.path.dirname(HERE), 'include', 'slipcam_b200.h'))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    """Compile the library if a source is newer than it (or force); returns its path."""
    if not force and not _stale():
        return LIB
    # one object per source, compiled side by side, then one link
    objs, procs = [], []
    for src in SOURCES:
        obj = os.path.join(CSRC, os.path.splitext(src)[0] + '.o')
        cmd = [NVCC, *FLAGS, '-c', os.path.join(CSRC, src), '-o', obj]
        if verbose:
            print(' '.join(cmd), flush=True)
        objs.append(obj)
        procs.append(subprocess.Popen(cmd))
    failed = [p.args for p in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    cmd = [NVCC, *LINK, *objs, '-o', LIB + '.tmp']
    if verbose:
        print(' '.join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    for obj in objs:
        os.remove(obj)
    os.replace(LIB + '.tmp', LIB)
    return LIB


if __name__ == '__main__':
    print(build(force='--force' in sys.argv, verbose=True))
