"""Autotuned launch shapes (srw_b200.tune, models/line_tuning.txt): the table is well formed and
holds only valid shapes; the library's tuning entry points validate what they are given; and on the
GPU every tuned shape gives the same field, bit for bit, as the built-in default shape (the shape
only moves lines between CTAs), so parity carries over to the tuned configurations."""
import ctypes as C
import os

import numpy as np
import pytest

from srw_b200 import capi, tune


def table():
    out = []
    if os.path.exists(tune.TXT):
        for line in open(tune.TXT):
            if line.startswith('#') or not line.strip():
                continue
            f = line.split()
            fam = tune.FAM_SPEC if (len(f) > 3 and f[3] == 'spec') or not tune.is_pow2(int(f[1])) else tune.FAM_POW2
            out.append((0 if f[0] == 'rows' else 1, int(f[1]), int(f[2]), fam))
    return out


def test_tuning_table_valid_shapes():
    t = table()
    lengths = set(tune.all_lengths(64, 16384))
    for axis, n, L, fam in t:
        assert n in lengths or (n & (n - 1)) == 0, n
        assert L in tune.candidates(axis, n, fam), (axis, n, L, fam)


def test_tuning_entry_points_validate():
    L = capi.lib()
    got = C.c_int()
    assert L.srwgTuneGetLines(0, 4096, C.byref(got)) == 0 and got.value >= 1
    assert L.srwgTuneGetLines(0, 1000, C.byref(got)) == 0 and got.value == 0      # no compile-time kernel
    assert L.srwgTuneSetLines(1, 4096, 3) != 0          # columns: a power of two
    assert L.srwgTuneSetLines(0, 4096, 64) != 0         # beyond shared memory / threads per CTA
    assert L.srwgTuneSetLines(2, 4096, 1) != 0
    assert L.srwgTuneSetLines(0, 2240, 2) == 0
    assert L.srwgTuneGetLines(0, 2240, C.byref(got)) == 0 and got.value == 2
    assert L.srwgTuneSetFamily(0, 2240, 1) != 0          # no power-of-two kernel for 2240
    assert L.srwgTuneSetFamily(1, 4096, 3) == 0          # the specialised kernel also serves 4096
    assert L.srwgTuneGetFamily(1, 4096, C.byref(got)) == 0 and got.value == 3
    assert L.srwgTuneSetLines(1, 4096, 4) != 0           # 4 x 256 threads: above its 512
    assert L.srwgTuneSetLines(1, 4096, 2) == 0
    assert L.srwgTuneSetFamily(1, 4096, 0) == 0 and L.srwgTuneGetFamily(1, 4096, C.byref(got)) == 0
    assert got.value == 1
    n = C.c_int()
    assert L.srwgTuneLoad(tune.TXT.encode() if os.path.exists(tune.TXT) else None, C.byref(n)) == 0


def test_pass_shapes_report_the_table():
    """tune.pass_shapes (the bench's record of the launch shapes) reports the family and lines per
    CTA of the packaged table's entries, valid shapes for every line pass, nothing for other passes."""
    L = capi.lib()
    n = C.c_int()
    assert L.srwgTuneLoad(tune.TXT.encode() if os.path.exists(tune.TXT) else None, C.byref(n)) == 0
    passes = [('resize', 1024, 1024, 1536, 1600), ('line_rows', 1536, 1600), ('line_cols', 1536, 1600),
              ('line_rows', 4096, 4096), ('line_cols', 4096, 4096)]
    got = tune.pass_shapes(passes)
    assert [g['pass'] for g in got] == ['line_rows 1536x1600', 'line_cols 1536x1600', 'line_rows 4096x4096',
                                        'line_cols 4096x4096']
    entries = {(axis, m): (lines, fam) for axis, m, lines, fam in table()}
    for g, (kind, nx, nz) in zip(got, passes[1:]):
        axis = 0 if kind == 'line_rows' else 1
        m = nx if axis == 0 else nz
        fam = tune.FAM_POW2 if g['family'] == 'pow2' else tune.FAM_SPEC
        assert g['lines_per_cta'] in tune.candidates(axis, m, fam), g
        if (axis, m) in entries:
            assert (g['lines_per_cta'], fam) == entries[(axis, m)], g


@pytest.mark.gpu
def test_tuned_shapes_give_identical_fields():
    torch = pytest.importorskip('torch')
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    t = table()
    if not t:
        pytest.skip('no tuning table')
    dev = torch.device('cuda', 0)
    L = capi.lib()
    try:
        for n in sorted({e[1] for e in t if e[1] <= 4096} | {1024, 4096}):
            outs = []
            for use_table in (False, True):
                if use_table:
                    assert L.srwgTuneLoad(tune.TXT.encode(), None) == 0
                else:
                    assert L.srwgTuneLoad(None, None) == 0
                p, ex = tune._plan(n, dev)
                a = torch.from_numpy(ex).to(dev)
                b = (a * 0.5j).contiguous()
                ox, oy = p.new_output()
                p.execute(a, b, ox, oy)
                torch.cuda.synchronize(dev)
                outs.append((ox.clone(), oy.clone()))
            assert torch.equal(outs[0][0], outs[1][0]) and torch.equal(outs[0][1], outs[1][1]), n
            assert float(outs[1][0].abs().max()) > 0
    finally:
        L.srwgTuneLoad(tune.TXT.encode() if os.path.exists(tune.TXT) else None, None)
