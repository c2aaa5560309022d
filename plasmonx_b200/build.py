"""Build the CUDA library in-tree: plasmonx_b200/libplasmonx_b200.so (sm_100a).

    python -m plasmonx_b200.build [--force]

nvcc compiles every ``csrc/*.cu`` for sm_100a and links one shared library
with a C ABI (``include/plasmonx_b200.h``); the cuSOLVER dense LU used by the
direct-inversion mode is linked from the CUDA toolkit.
"""
import glob
import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, 'libplasmonx_b200.so')
NVCC = os.environ.get('NVCC', '/usr/local/cuda/bin/nvcc')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
FLAGS = ['-O3', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC', '--expt-relaxed-constexpr']


def sources():
    return sorted(glob.glob(os.path.join(HERE, 'csrc', '*.cu')))


def _digest():
    h = hashlib.sha256()
    for p in sources() + sorted(glob.glob(os.path.join(HERE, 'csrc', '*.h*'))) + \
            sorted(glob.glob(os.path.join(HERE, 'csrc', '*.cuh'))) + \
            [os.path.join(ROOT, 'include', 'plasmonx_b200.h'), os.path.abspath(__file__)]:
        with open(p, 'rb') as f:
            h.update(p.encode() + f.read())
    return h.hexdigest()


def build(force=False, verbose=False):
    stamp = LIB + '.sha256'
    dig = _digest()
    if not force and os.path.exists(LIB) and os.path.exists(stamp):
        with open(stamp) as f:
            if f.read().strip() == dig:
                return LIB
    objdir = os.path.join(HERE, '_build')
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + '.o')
        cmd = [NVCC, *ARCH, *FLAGS, '-I', os.path.join(ROOT, 'include'), '-c', src, '-o', obj]
        if verbose:
            print(' '.join(cmd))
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
    errs = []
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            errs.append('%s:\n%s' % (src, out.decode()))
        elif verbose and out:
            print(out.decode())
    if errs:
        raise RuntimeError('nvcc failed\n' + '\n'.join(errs))
    tmp = LIB + '.tmp'
    cmd = [NVCC, *ARCH, '-shared', '-o', tmp, *objs, '-lcusolver', '-lcublas', '-lcudart']
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    with open(stamp, 'w') as f:
        f.write(dig)
    return LIB


if __name__ == '__main__':
    print(build(force='--force' in sys.argv, verbose='-v' in sys.argv))
