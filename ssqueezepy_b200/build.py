# -*- coding: utf-8 -*-
"""Build the CUDA extension in-tree: ssqueezepy_b200/_lib/libssqb.so.

nvcc compiles each csrc/*.cu for sm_100a (compute_100a SASS) in parallel and
links one shared library exporting the C ABI of include/ssqb.h, with the CUDA
runtime linked statically so the library has no runtime-version coupling to
the Python environment.

    python -m ssqueezepy_b200.build [--force] [-j N]
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
LIBDIR = os.path.join(HERE, '_lib')
LIB = os.path.join(LIBDIR, 'libssqb.so')
INCLUDE = os.path.join(os.path.dirname(HERE), 'include')
OBJDIR = os.path.join(HERE, '_build')

NVCC = os.environ.get('NVCC', '/usr/local/cuda/bin/nvcc')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
FLAGS = ['-std=c++17', '-O3', '-lineinfo', '-Xcompiler', '-fPIC',
         '-Xcompiler', '-fvisibility=hidden', '--expt-relaxed-constexpr']


def _sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC)
                  if f.endswith('.cu'))


def _deps():
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    files.append(os.path.join(INCLUDE, 'ssqb.h'))
    files.append(os.path.abspath(__file__))
    return files


def _includes(src, seen=None):
    """`src` and the files it includes with quoted #include, recursively."""
    import re
    seen = set() if seen is None else seen
    src = os.path.abspath(src)
    if src in seen or not os.path.exists(src):
        return seen
    seen.add(src)
    with open(src) as f:
        for m in re.finditer(r'^\s*#include\s+"([^"]+)"', f.read(), re.M):
            _includes(os.path.join(os.path.dirname(src), m.group(1)), seen)
    return seen


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in _deps())


def build(force=False, jobs=None, verbose=False):
    if not force and up_to_date():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(OBJDIR, exist_ok=True)
    srcs = _sources()

    # an object is reused when it is newer than its source, than every
    # header it includes (followed through quoted #include lines) and than
    # this script; otherwise it is rebuilt
    def compile_one(src):
        obj = os.path.join(OBJDIR, os.path.basename(src)[:-3] + '.o')
        t_dep = max(os.path.getmtime(f) for f in _includes(src))
        if (not force and os.path.exists(obj)
                and os.path.getmtime(obj) >= max(t_dep, os.path.getmtime(__file__))):
            return obj
        cmd = [NVCC, *ARCH, *FLAGS, '-I', INCLUDE, '-c', src, '-o', obj]
        if verbose:
            cmd.insert(1, '-Xptxas=-v')
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError('nvcc failed for %s:\n%s%s'
                               % (src, r.stdout, r.stderr))
        if verbose:
            sys.stderr.write(r.stderr)
        return obj

    with ThreadPoolExecutor(jobs or min(len(srcs), os.cpu_count() or 1)) as ex:
        objs = list(ex.map(compile_one, srcs))
    tmp = LIB + '.tmp'
    cmd = [NVCC, *ARCH, '-shared', '-cudart', 'static', '-o', tmp, *objs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError('link failed:\n%s%s' % (r.stdout, r.stderr))
    os.replace(tmp, LIB)
    return LIB


if __name__ == '__main__':
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument('--force', action='store_true')
    ap.add_argument('-j', type=int, default=None)
    ap.add_argument('-v', action='store_true')
    a = ap.parse_args()
    print(build(force=a.force, jobs=a.j, verbose=a.v))
