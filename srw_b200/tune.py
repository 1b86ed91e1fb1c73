"""Autotuner of the FFT line passes' launch shapes (the reference has none: FFTW plans per call,
gmfft.cpp:295; its CUDA build caches cuFFT plans, gmfft.h:182-187).

For every line length with a compile-time kernel (powers of two and the general lengths of
csrc/linen_lengths.h) it times the two passes of an N x N propagation to the waist (a row pass and
a column pass, the headline beamline's FFT) for every valid kernel family (powers of two: the
power-of-two pass or the specialised pass) and number of lines per CTA of each pass -- which is
also the CTA size and, for the column pass, the width of the column blocks the row pass writes --
with CUDA events on the launching stream and L2 flushed between repetitions, keeps the fastest
pair and writes

  models/line_tuning.txt    "rows|cols N L [spec]" lines, read by the library at its first plan
  models/line_tuning.json   every measurement (ms per pass), read by the learned-factor cost model

    python -m srw_b200.tune [--lengths 1280,2240] [--reps 7]          # GPU

torch supplies device memory, streams and events only.
"""
import argparse
import ctypes as C
import json
import os
import re
import time

import numpy as np

from . import capi

HERE = os.path.dirname(os.path.abspath(__file__))
TXT = os.path.join(HERE, 'models', 'line_tuning.txt')
JSN = os.path.join(HERE, 'models', 'line_tuning.json')
LENGTHS_H = os.path.join(HERE, 'csrc', 'linen_lengths.h')
SMEM_MAX = 220 * 1024


def general_lengths():
    txt = open(LENGTHS_H).read()
    block = txt[txt.index('SRWG_LINEN_LENGTHS(X)'):txt.index('SRWG_LINEN_POW2(X)')]
    return [int(v) for v in re.findall(r'X\((\d+)\)', block)]


def all_lengths(lo=256, hi=8192):
    p2 = [1 << k for k in range(8, 14) if lo <= (1 << k) <= hi]
    return sorted(set(p2 + [n for n in general_lengths() if lo <= n <= hi]))


def is_pow2(n):
    return n & (n - 1) == 0


FAM_POW2, FAM_SPEC = 1, 3          # kernel families: power-of-two pass, specialised pass


def line_pitch(n, lines=1, cols=False):
    """The library's shared-memory pitch of a line (kernels.h line_pitch)."""
    p = n + n // 16
    r = (1 if lines >= 16 else 16 // lines) if (cols and lines >= 2) else 4
    return p + (r + 16 - p % 16) % 16
POW2_SPEC = [256, 512, 1024, 2048, 4096, 8192]       # powers of two the specialised pass is built for


def families(n):
    if is_pow2(n):
        return [FAM_POW2] + ([FAM_SPEC] if n in POW2_SPEC else [])
    return [FAM_SPEC]


def launch_shape(axis, n):
    """(kernel family name, lines per CTA) the library uses for a line pass of n points along axis 0
    (rows) or 1 (columns): the tuning table's entry, else its defaults; (None, 0) for lengths that
    run the run-time-scheduled pass."""
    L = capi.lib()
    fam, lines = C.c_int(), C.c_int()
    capi.check(L.srwgTuneGetFamily(int(axis), int(n), C.byref(fam)), 'tune family')
    capi.check(L.srwgTuneGetLines(int(axis), int(n), C.byref(lines)), 'tune lines')
    name = {FAM_POW2: 'pow2', FAM_SPEC: 'spec'}.get(fam.value)
    return name, (lines.value if name else 0)


def pass_shapes(passes):
    """Launch shapes of the line passes of a plan (Plan.kernels() / MultiE.info() tuples)."""
    out = []
    for k in passes:
        if k[0] in ('line_rows', 'line_cols'):
            axis = 0 if k[0] == 'line_rows' else 1
            fam, lines = launch_shape(axis, k[1] if axis == 0 else k[2])
            out.append({"pass": "%s %dx%d" % (k[0], k[1], k[2]), "family": fam, "lines_per_cta": lines})
    return out


def candidates(axis, n, fam=None):
    """Valid (family, lines per CTA) pairs (the library's fixed_lines_valid): shared memory, threads
    per CTA (1024 for the power-of-two pass, 512 for the specialised one), columns a power of two up
    to 32; `fam` restricts them to one family (then plain lines per CTA are returned)."""
    out = []
    for f in families(n) if fam is None else [fam]:
        t = n // 16 if f == FAM_POW2 else (n + 15) // 16
        tmax = 1024 if f == FAM_POW2 else 512
        for L in range(1, 33):
            if L * line_pitch(n, L, axis == 1) * 8 > SMEM_MAX or t * L > tmax:
                break
            if axis == 1 and (L & (L - 1)):
                continue
            if axis == 0 and L > 8:
                break
            out.append(L if fam is not None else (f, L))
    return out


def _plan(n, dev):
    """N x N Gaussian (2 keV, curved) through a 10 m drift to the waist: one row and one column pass."""
    from . import srwlib as S
    from .plan import Plan
    r = 1.5e-3
    w = S.SRWLWfr()
    w.allocate(1, n, n)
    x = np.linspace(-r, r, n)
    X, Y = np.meshgrid(x, x)
    ex = (np.exp(-(X * X + Y * Y) / (4. * (0.4e-3) ** 2)) * 1e6).astype(np.complex64)
    a = np.empty(2 * n * n, np.float32)
    a[0::2], a[1::2] = ex.real.ravel(), ex.imag.ravel()
    w.arEx, w.arEy = a, a.copy()
    w.mesh.xStart, w.mesh.xFin, w.mesh.yStart, w.mesh.yFin = -r, r, -r, r
    w.mesh.eStart = w.mesh.eFin = 2012.
    w.Rx = w.Ry = 20.
    w.dRx = w.dRy = 0.2
    opt = S.SRWLOptC([S.SRWLOptD(10.)], [[0, 0, 1., 4, 0, 1., 1., 1., 1., 0, 0, 0]])
    return Plan(w, opt, device=dev.index), ex


def time_passes(n, cr, cc, dev, reps=7, flush=None):
    """Median CUDA-event time [ms] of the row and the column pass with the (family, lines per CTA)
    pairs cr / cc."""
    import torch
    L = capi.lib()
    capi.check(L.srwgTuneSetFamily(0, n, cr[0]), 'tune rows')
    capi.check(L.srwgTuneSetLines(0, n, cr[1]), 'tune rows')
    capi.check(L.srwgTuneSetFamily(1, n, cc[0]), 'tune cols')
    capi.check(L.srwgTuneSetLines(1, n, cc[1]), 'tune cols')
    p, ex = _plan(n, dev)
    kinds = [k[0] for k in p.kernels()]
    if kinds != ['line_rows', 'line_cols']:
        raise RuntimeError('unexpected passes %s' % kinds)
    a = torch.from_numpy(ex).to(dev)
    b = a.clone()
    ox, oy = p.new_output()
    st = torch.cuda.current_stream(dev)
    for _ in range(2):
        p.execute(a, b, ox, oy)
    ms = []
    for _ in range(reps):
        if flush is not None:
            flush.fill_(1)
        ms.append(p.execute_timed(a, b, ox, oy, st))
    torch.cuda.synchronize(dev)
    m = np.median(np.array(ms), 0)
    return float(m[0]), float(m[1])


def tune(lengths, dev, reps=7, log=print, on_length=None):
    import torch
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)      # > L2 (126 MB)
    L = capi.lib()
    res = {}
    for n in lengths:
        t0 = time.time()
        rows_c, cols_c = candidates(0, n), candidates(1, n)
        meas = []
        for cc in cols_c:
            for cr in rows_c:
                tr, tc = time_passes(n, cr, cc, dev, reps, flush)
                meas.append((cr, cc, tr, tc))
        # defaults (the library's own choice without a table entry), for the record
        for ax in (0, 1):
            capi.check(L.srwgTuneSetLines(ax, n, 0), 'tune')
        d = [C.c_int() for _ in range(4)]
        L.srwgTuneGetFamily(0, n, C.byref(d[0]))
        L.srwgTuneGetLines(0, n, C.byref(d[1]))
        L.srwgTuneGetFamily(1, n, C.byref(d[2]))
        L.srwgTuneGetLines(1, n, C.byref(d[3]))
        dr, dc = (d[0].value, d[1].value), (d[2].value, d[3].value)
        dflt = next((m for m in meas if m[0] == dr and m[1] == dc), None)
        best = min(meas, key=lambda m: m[2] + m[3])
        res[n] = dict(rows=best[0][1], rows_family=best[0][0], cols=best[1][1], cols_family=best[1][0],
                      rows_ms=best[2], cols_ms=best[3], default=[list(dr), list(dc)],
                      default_ms=[dflt[2], dflt[3]] if dflt else None,
                      measured=[[list(m[0]), list(m[1]), m[2], m[3]] for m in meas])
        log('N %5d  best rows %s %.4f ms  cols %s %.4f ms  (default %s / %s: %s)  %.1f s' % (
            n, best[0], best[2], best[1], best[3], dr, dc,
            '%.4f + %.4f ms' % (dflt[2], dflt[3]) if dflt else '-', time.time() - t0))
        if on_length is not None:
            on_length(res)
    return res


def write(res, txt=TXT, jsn=JSN, device_name=''):
    os.makedirs(os.path.dirname(txt), exist_ok=True)
    with open(txt, 'w') as f:
        f.write('# lines per CTA of the line passes with compile-time lengths, measured by srw_b200.tune\n')
        f.write('# on %s (row + column pass of an N x N propagation to the waist, median CUDA-event time)\n'
                % device_name)
        for n in sorted(res):
            r = res[n]
            for ax in ('rows', 'cols'):
                spec = ' spec' if (is_pow2(n) and r[ax + '_family'] == FAM_SPEC) else ''
                f.write('%s %d %d%s\n' % (ax, n, r[ax], spec))
    with open(jsn, 'w') as f:
        json.dump({'device': device_name, 'lengths': {str(n): res[n] for n in sorted(res)}}, f, indent=0)


def load_times(jsn=JSN):
    """{N: (rows ms, cols ms)} of the tuned launch shapes, or {} without a table."""
    if not os.path.exists(jsn):
        return {}
    d = json.load(open(jsn))
    return {int(n): (v['rows_ms'], v['cols_ms']) for n, v in d.get('lengths', {}).items()}


def main():
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument('--lengths', default='')
    ap.add_argument('--reps', type=int, default=7)
    ap.add_argument('--txt', default=TXT)
    ap.add_argument('--json', default=JSN)
    args = ap.parse_args()
    dev = torch.device('cuda', 0)
    lengths = [int(v) for v in args.lengths.split(',') if v] or all_lengths()
    capi.lib().srwgTuneLoad(None, None)            # measure from the built-in defaults
    name = torch.cuda.get_device_name(dev)
    # the table is rewritten after every length, so that an interrupted run keeps what it measured
    res = tune(lengths, dev, args.reps, on_length=lambda r: write(r, args.txt, args.json, name))
    write(res, args.txt, args.json, name)
    print('wrote %s, %s' % (args.txt, args.json))


if __name__ == '__main__':
    main()
