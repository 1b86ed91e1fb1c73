"""CPU tests of the C-ABI library: it loads, exports every entry point declared in include/*.h,
and its host planner reproduces the reference's meshes and wavefront scalars bit-exactly (the
planning half of srwlPropagElecField runs without a GPU)."""
import os
import re

import numpy as np
import pytest

from srw_b200 import capi
from srw_b200.plan import Plan
from tests.golden_cases import STAGED, case_io, load
from tests.helpers import beamline, gaussian, make_wfr, C1, C1PP, PP

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
D, INDEX = load()


def header_symbols():
    names = []
    inc = os.path.join(REPO, 'include')
    for f in os.listdir(inc):
        if f.endswith('.h'):
            names += re.findall(r'SRWG_API\s+[\w\s\*]+?\b(\w+)\s*\(', open(os.path.join(inc, f)).read())
    return names


def test_library_exports_every_declared_symbol():
    L = capi.lib()
    names = header_symbols()
    assert 'srwlPropagElecField' in names and 'srwgPlanExecute' in names
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(capi.SYMBOLS), set(names) ^ set(capi.SYMBOLS)


def test_error_texts():
    assert 'callback' in capi.err_text(23172)
    assert 'one point' in capi.err_text(23059)


def plan_case(name):
    c = next(c for c in INDEX if c['name'] == name)
    i, o = case_io(D, name)
    w = make_wfr(i['ex'], i['ey'], i['mesh'], i['Rx'], i['Ry'], i['dRx'], i['dRy'], i['xc'], i['yc'],
                 i['momX'], i['momY'], propM=i['prop'])
    return Plan(w, beamline(c['elements'], c['props'])), o


def plan_prop_matrix(p):
    """arElecPropMatr of a plan's output (the 4x4 propagation matrix and vector)."""
    import ctypes as C
    from srw_b200 import capi
    out = capi.SRWLWfr()
    m = np.zeros(20)
    out.arElecPropMatr = m.ctypes.data
    assert capi.lib().srwgPlanGetOutput(p._h, C.byref(out)) == 0
    return m


@pytest.mark.parametrize('name', [c['name'] for c in INDEX])
def test_planner_mesh_bit_exact(name):
    if name in STAGED:      # the plan depends on moments measured from the field: refused here
        with pytest.raises(RuntimeError, match='plans in stages'):
            plan_case(name)
        return
    p, o = plan_case(name)
    np.testing.assert_allclose(plan_prop_matrix(p), o['prop'], rtol=1e-14, atol=1e-300)
    m = p.output_mesh()
    mine = np.array([m['nx'], m['ny'], m['xStart'], m['xFin'], m['yStart'], m['yFin']])
    assert np.array_equal(mine, o['mesh_raw']), (mine, o['mesh_raw'])
    assert [m['Rx'], m['Ry'], m['dRx'], m['dRy'], m['xc'], m['yc']] == [o['Rx'], o['Ry'], o['dRx'], o['dRy'], o['xc'], o['yc']]


def test_pass_fusion_counts():
    # C0: 2 angular drifts around aperture+lens -> 5 passes, but the aperture clips the beam: the
    # moments are measured on the masked field (a moment pass), so the lens starts a new row pass
    # -> 6 field passes + 1 moment pass; C1: resize (+ the aperture and the quadratic-term removal
    # before it, + the lens after it), to-waist rows + columns -> 3
    k = [x[0] for x in plan_case('c0_64')[0].kernels()]
    assert len(k) == 7 and k.count('moments') == 1 and k.index('moments') == 3
    assert plan_case('c1_64')[0].n_kernels == 3
    assert plan_case('c2_128')[0].n_kernels == 5


def test_full_size_c1_plan():
    ex, ey, mesh = gaussian(1024, E=2000., sig=0.4e-3, r=1.5e-3)
    w = make_wfr(ex, ey, mesh, Rx=20., Ry=20., dRx=0.2, dRy=0.2)
    p = Plan(w, beamline(C1, C1PP))
    assert (p.nx_out, p.ny_out) == (4096, 4096)
    k = p.kernels()
    assert k[0][0] == 'resize' and k[0][3:] == (4096, 4096)
    assert 'pre=1' in p.describe() and 'tile=' in p.describe()


def test_aperture_bounds_the_resize_window():
    """The undulator beamline's circular aperture (0.8 mm, folded into the resize before the lens)
    bounds the resize window: the new points whose 4-point stencils reach the aperture's box (its
    radius in old steps, widened by 2 nodes against coordinate rounding, plus the stencil), not the
    whole old range; the row pass transforms only those rows and does not write the others, and the
    column pass loads only that window of every column."""
    import re
    ex, ey, mesh = gaussian(1024, E=2000., sig=0.4e-3, r=1.5e-3)
    w = make_wfr(ex, ey, mesh, Rx=20., Ry=20., dRx=0.2, dRy=0.2)
    d = Plan(w, beamline(C1, C1PP)).describe().splitlines()
    x0, x1, z0, z1 = map(int, re.search(r'window=x(\d+):(\d+),z(\d+):(\d+)', d[0]).groups())
    step_old, step_new = 3e-3 / 1023, 6e-3 / 4095          # range x2, resolution x2
    r = 0.4e-3
    half_old = int(np.ceil(r / step_old)) + 2 + 1             # aperture box half-width in old nodes (+ margin)
    half_new = (half_old + 2) * step_old / step_new           # ... and the stencil reach, in new steps
    assert (x0, x1) == (z0, z1)
    assert abs((x1 - x0) / 2. - half_new) < 4 and x1 - x0 < 4096 // 4
    assert abs((x0 + x1) / 2. - 2047.5) <= 1.
    assert 'lines=%d:%d points=%d:%d' % (z0, z1, x0, x1) in d[1]
    assert 'lines=0:4095 points=%d:%d' % (z0, z1) in d[2]


def test_unsupported_and_invalid_inputs_raise():
    ex, ey, mesh = gaussian(64)
    w = make_wfr(ex, ey, mesh)
    with pytest.raises(RuntimeError, match='pp\\[3\\]=100'):
        Plan(w, beamline([('drift', 1., 0)], [PP(100)]))
    with pytest.raises(RuntimeError, match='automatic resizing'):
        Plan(w, beamline([('drift', 1., 0)], [[1, 0, 1., 0, 0, 1., 1., 1., 1.]]))
    ex1, ey1, mesh1 = gaussian(64, ny=1)
    with pytest.raises(RuntimeError, match='one point'):
        Plan(make_wfr(ex1, ey1, mesh1), beamline([('drift', 1., 0)], [PP()]))

    class SRWLOptMirEl(object):
        pass
    from srw_b200.srwlib import SRWLOptC, SRWLOptT
    with pytest.raises(RuntimeError, match='not supported'):
        Plan(w, SRWLOptC([SRWLOptMirEl()], [PP()]))
    # a transmission table without its data is refused
    bad = SRWLOptT(8, 8, 1e-3, 1e-3)
    bad.arTr = None
    with pytest.raises(RuntimeError, match='Transmission'):
        Plan(w, SRWLOptC([bad], [PP()]))
