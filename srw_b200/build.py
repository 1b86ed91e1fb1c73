"""Builds the CUDA library in-tree: srw_b200/_lib/libsrwl_b200.so (sm_100a).

    python -m srw_b200.build          # or srw_b200.build.build()
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
OUT_DIR = os.path.join(HERE, '_lib')
OBJ_DIR = os.path.join(HERE, '_build')          # objects: kept out of the shipped tree
LIB = os.path.join(OUT_DIR, 'libsrwl_b200.so')
NVCC = os.environ.get('NVCC', '/usr/local/cuda/bin/nvcc')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
SOURCES = ['kernels.cu'] + ['line2_%d.cu' % l for l in range(6, 15)] + ['line2e_%d.cu' % l for l in range(6, 15)] + ['planner.cpp', 'tables.cpp', 'capi.cpp', 'noalloc.cu', 'lineg.cu', 'lineg_e.cu', 'multie.cu', 'mlp.cu', 'moments.cu', 'intensity.cu', 'gaussian.cu']

def linen_lengths():
    """Lengths of the specialised general-length line kernels (csrc/linen_lengths.h)."""
    import re
    txt = open(os.path.join(CSRC, 'linen_lengths.h')).read()
    return sorted(set(int(v) for v in re.findall(r'X\((\d+)\)', txt)))


# host code: no FP contraction so the mesh bookkeeping rounds exactly like the reference
HOST_FLAGS = '-O2,-fPIC,-ffp-contract=off,-fvisibility=hidden'


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(' '.join(cmd) + '\n' + r.stdout + r.stderr)
        raise RuntimeError('build step failed: ' + os.path.basename(cmd[-1]))
    return r.stdout + r.stderr


def _includes(path, seen):
    """The source and every project header it includes, transitively (quoted includes)."""
    if path in seen or not os.path.exists(path):
        return seen
    seen.add(path)
    with open(path) as f:
        for line in f:
            t = line.strip()
            if t.startswith('#include "'):
                _includes(os.path.normpath(os.path.join(os.path.dirname(path), t.split('"')[1])), seen)
    return seen


def _compile(s, ptxas_info):
    defs = []
    if '@' in s:                      # linen.cu@N: the specialised general-length pass for N points
        s, n = s.split('@')
        defs = ['-DSRWG_LINEN=' + n]
        obj = os.path.join(OBJ_DIR, 'linen_%s.cu.o' % n)
    else:
        obj = os.path.join(OBJ_DIR, s + '.o')
    src = os.path.join(CSRC, s)
    deps = sorted(_includes(src, set()))
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(d) for d in deps) and not ptxas_info:
        return obj, ''
    cmd = [NVCC, '-c', '-O3', '-std=c++17', '-lineinfo', '-Xcompiler', HOST_FLAGS, '--fmad=true'] + ARCH + \
          defs + ['-I', CSRC, '-o', obj, src]
    if ptxas_info and s.endswith('.cu'):
        cmd.insert(1, '-Xptxas=-v')
    return obj, _run(cmd)


def build(verbose=False, ptxas_info=False):
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(OUT_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    units = SOURCES + ['linen.cu@%d' % n for n in linen_lengths()]
    # longest units first, so that the pool's last wave is short
    units.sort(key=lambda u: (not u.startswith('line2'), u))
    with ThreadPoolExecutor(max_workers=max(1, min(len(units), os.cpu_count() or 1))) as ex:
        res = list(ex.map(lambda s: _compile(s, ptxas_info), units))
    objs = [o for o, _ in res]
    if verbose or ptxas_info:
        for _, out in res:
            sys.stdout.write(out)
    # exported symbols: the C-ABI in include/srwl_b200.h
    _run([NVCC, '-shared', '-o', LIB] + ARCH + objs + ['-lcudart'])
    return LIB


if __name__ == '__main__':
    print(build(verbose=True, ptxas_info='-v' in sys.argv))
