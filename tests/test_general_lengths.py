"""General FFT lengths (2^a 3^b 5^c 7^d): the specialised line kernels (linen.cuh, one per length of
linen_lengths.h) and the run-time-scheduled one, against the FP64 oracle through the C-ABI.  Bar as
the other parity tests: meshes bit-exact, field and intensity within relative L2 1e-4."""
import os
import re

import numpy as np
import pytest

from tests.helpers import C0PP, C1, PP, beamline, fields, gaussian, make_wfr, mesh_tuple, oracle_run, rel_l2

TOL = 1e-4
HERE = os.path.dirname(os.path.abspath(__file__))
LENGTHS_H = os.path.join(os.path.dirname(HERE), 'srw_b200', 'csrc', 'linen_lengths.h')


def linen_lengths():
    txt = open(LENGTHS_H).read()
    block = txt[txt.index('SRWG_LINEN_LENGTHS(X)'):txt.index('SRWG_LINEN_POW2(X)')]
    return [int(v) for v in re.findall(r'X\((\d+)\)', block)]


def schedule(n):
    """The kernels' compile-time radix schedule (linen.cuh nsched), restated."""
    m, p2, r = n, 0, []
    while m % 2 == 0:
        m //= 2
        p2 += 1
    while p2 >= 4:
        r.append(16)
        p2 -= 4
    if p2:
        r.append(1 << p2)
    for p in (3, 5, 7):
        while m % p == 0:
            r.append(p)
            m //= p
    return r if m == 1 else None


def test_specialised_lengths_have_valid_schedules():
    ls = linen_lengths()
    assert len(ls) == len(set(ls)) and ls == sorted(ls)
    for n in ls:
        r = schedule(n)
        assert r is not None and 2 <= len(r) <= 8, n
        assert int(np.prod(r)) == n
        assert n % 16 == 0 and (n & (n - 1)) != 0          # 16 points per thread; powers of two go to line2
        p = n + n // 16
        p += (4 + 16 - p % 16) % 16                         # the library's line pitch
        assert p % 16 == 4 and p >= n + n // 16 and p * 8 <= 220 * 1024


# ------------------------------------------------------------------------------------------------
# GPU
# ------------------------------------------------------------------------------------------------
def _gpu():
    torch = pytest.importorskip('torch')
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')


def _families(ex, ey, mesh, el, pp, sc):
    from srw_b200.plan import Plan
    p = Plan(make_wfr(ex, ey, mesh, **sc), beamline(el, pp))
    return [l.split('fft=')[1].split()[0] for l in p.describe().splitlines() if ' LINE ' in l]


def _check(ex, ey, mesh, el, pp, sc, want_family='spec'):
    from srw_b200 import srwlpy as srwl
    fam = _families(ex, ey, mesh, el, pp, sc)
    assert want_family in fam, fam
    w = make_wfr(ex, ey, mesh, **sc)
    srwl.PropagElecField(w, beamline(el, pp))
    o = oracle_run(ex, ey, mesh, el, pp, **sc)
    m = o.out_mesh()
    assert np.array_equal(mesh_tuple(w), np.array([m['nx'], m['ny'], m['xStart'], m['xFin'], m['yStart'], m['yFin']]))
    gx, gy = fields(w)
    assert rel_l2(gx, o.ex) < TOL
    if np.linalg.norm(o.ey) > 0:
        assert rel_l2(gy, o.ey) < TOL
    assert rel_l2(np.abs(gx) ** 2 + np.abs(gy) ** 2, np.abs(o.ex) ** 2 + np.abs(o.ey) ** 2) < TOL
    return w


@pytest.mark.gpu
@pytest.mark.parametrize('n,rf,df', [(256, 1.25, 1.75), (256, 1.5, 1.), (256, 1.25, 1.25), (512, 1.75, 1.),
                                     (512, 1.5, 1.5), (512, 1.25, 1.5), (1024, 1.25, 1.75), (1024, 1.5, 1.)])
def test_resize_lens_to_waist(n, rf, df):
    """The undulator beamline (aperture, resize (rf, df) before the lens, drift to the waist) on
    grids of general length: one forward transform per pass, centring rotations, the to-waist
    factors, column blocks and zero windows."""
    _gpu()
    ex, _, mesh = gaussian(n, E=2012., sig=0.35e-3, r=1.5e-3, R=20.)
    ey = 0.05j * ex
    _check(ex, ey, mesh, C1, [PP(), PP(0, rf, df, rf, df), PP(4)], dict(Rx=20., Ry=20., dRx=0.2, dRy=0.2))


@pytest.mark.gpu
@pytest.mark.parametrize("nx,ny", [(320, 448), (2240, 1536), (560, 384)])
def test_angular_drifts_ragged(nx, ny):
    """Angular-representation drifts (two transforms per pass, forward then inverse, transfer
    function and its quartic term between them), a circular aperture and a lens on ragged meshes of
    general lengths."""
    _gpu()
    ex, ey, mesh = gaussian(nx, E=1000., sig=50e-6, r=1e-3, ny=ny, ry=0.9e-3)
    el = [('drift', 10., 0), ('aperture', 'c', 'a', 1.2e-3, 1.2e-3, 0.05e-3, 0.), ('lens', 5., 5., 0., 0.),
          ('drift', 5., 0)]
    _check(ex, ey, mesh, el, C0PP, {})


@pytest.mark.gpu
def test_quadratic_phase_drifts_general_length():
    """Quadratic-phase analytic drifts (pp[3] = 2) with the lens between them at 1280^2 (mirror of
    the field where the magnification is negative)."""
    _gpu()
    ex, ey, mesh = gaussian(1280, E=10000., sig=20e-6, r=1e-3, R=30.)
    el = [('drift', 30., 0), ('lens', 15., 15., 0., 0.), ('drift', 30., 0)]
    _check(ex, ey, mesh, el, [PP(2), PP(), PP(2)], dict(Rx=30., Ry=30., dRx=0.3, dRy=0.3))


@pytest.mark.gpu
def test_runtime_scheduled_length_still_works():
    """Lengths outside the specialised list (216 = 2^3 3^3 and 200 = 2^3 5^2: fewer than 16 points per
    thread) run the run-time-scheduled kernel, against the oracle."""
    _gpu()
    ex, ey, mesh = gaussian(216, E=1000., sig=50e-6, r=1e-3, ny=200, ry=1e-3)
    el = [('drift', 10., 0), ('lens', 5., 5., 0., 0.), ('drift', 5., 0)]
    _check(ex, ey, mesh, el, [PP()] * 3, {}, want_family='gen')


@pytest.mark.gpu
def test_bulk_copy_wait_limit_reports_and_recovers():
    """The specialised passes wait for the bulk copies of their input tiles with an iteration limit.
    With the limit at one try the waits give up: the library counts them (srwgGetWaitStatus) and the
    CTAs skip their work, with no fault; with the default limit the same propagation is exact again
    and counts nothing."""
    _gpu()
    import ctypes as C
    from srw_b200 import capi
    from srw_b200 import srwlpy as srwl
    L = capi.lib()
    ex, _, mesh = gaussian(1024, E=2012., sig=0.35e-3, r=1.5e-3, R=20.)
    ey = 0.05j * ex
    el, pp, sc = C1, [PP(), PP(0, 1., 1.25, 1., 1.25), PP(4)], dict(Rx=20., Ry=20., dRx=0.2, dRy=0.2)
    assert 'spec' in _families(ex, ey, mesh, el, pp, sc)
    n = C.c_int()
    try:
        assert L.srwgGetWaitStatus(0, C.byref(n), 1) == 0
        assert L.srwgSetWaitLimit(1) == 0
        w = make_wfr(ex, ey, mesh, **sc)
        srwl.PropagElecField(w, beamline(el, pp))
        assert L.srwgGetWaitStatus(0, C.byref(n), 1) == 0
        assert n.value > 0
    finally:
        L.srwgSetWaitLimit(0)
    w = _check(ex, ey, mesh, el, pp, sc)
    assert L.srwgGetWaitStatus(0, C.byref(n), 1) == 0 and n.value == 0
