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
SOURCES = ['capi.cu']
NVCC = os.environ.get('NVCC', '/usr/local/cuda/bin/nvcc')
FLAGS = ['-std=c++17', '-O3', '--expt-relaxed-constexpr', '-gencode', 'arch=compute_100a,code=sm_100a',
         '-lineinfo', '-Xcompiler', '-fPIC', '-Xcompiler', '-fvisibility=hidden', '-shared',
         '-cudart', 'static', '-diag-suppress', '20014']


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
    cmd = [NVCC, *FLAGS, *[os.path.join(CSRC, s) for s in SOURCES], '-o', LIB + '.tmp']
    if verbose:
        print(' '.join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(LIB + '.tmp', LIB)
    return LIB


if __name__ == '__main__':
    print(build(force='--force' in sys.argv, verbose=True))
