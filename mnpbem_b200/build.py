"""Build the CUDA library ``mnpbem_b200/libmnpbem_b200.so`` for sm_100a.

    python -m mnpbem_b200.build [--force] [--verbose]

Each ``csrc/*.cu`` is compiled by nvcc into ``_build/`` (in parallel) and
linked into one shared library next to this file, so the library travels with
the source tree.  Objects are rebuilt when the source or any header is newer.
"""

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, 'csrc')
BUILD = os.path.join(ROOT, '_build')
LIB = os.path.join(HERE, 'libmnpbem_b200.so')

ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
NVCC_FLAGS = ['-O3', '-lineinfo', '-std=c++17', '--expt-relaxed-constexpr',
              '-Xcompiler', '-fPIC', '-Xcompiler', '-ffp-contract=off',
              '-I' + os.path.join(ROOT, 'include')]


def nvcc():
    for cand in (os.environ.get('NVCC'), shutil.which('nvcc'), '/usr/local/cuda/bin/nvcc'):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newest_header():
    hs = glob.glob(os.path.join(CSRC, '*.cuh')) + glob.glob(os.path.join(ROOT, 'include', '*.h'))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src, force, verbose, extra):
    obj = os.path.join(BUILD, os.path.basename(src) + '.o')
    if (not force and os.path.exists(obj) and
            os.path.getmtime(obj) >= max(os.path.getmtime(src), _newest_header())):
        return obj, None
    cmd = [nvcc()] + ARCH + NVCC_FLAGS + extra + ['-c', src, '-o', obj]
    if verbose:
        print(' '.join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, r.stdout + r.stderr
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)
    return obj, None


def build(force=False, verbose=False, ptxas_info=False):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, '*.cu')))
    extra = ['-Xptxas', '-v'] if ptxas_info else []
    objs, errors = [], []
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        for obj, err in ex.map(lambda s: _compile(s, force or ptxas_info, verbose, extra), srcs):
            objs.append(obj)
            if err:
                errors.append(err)
    if errors:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errors))
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [nvcc()] + ARCH + ['-shared', '-o', LIB] + objs + ['-lcudart']
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    return LIB


if __name__ == '__main__':
    lib = build(force='--force' in sys.argv, verbose='--verbose' in sys.argv,
                ptxas_info='--ptxas' in sys.argv)
    print(lib)
