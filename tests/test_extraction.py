"""Intensities extracted during propagation (srwlPropagElecField's nInt / arID / arIM / arI,
srTCompositeOptElem::ExtractPropagatedIntensity, cpp/src/core/sroptcnt.cpp:429): the oracle's
per-element states against the reference's extractions (golden fixtures), the Python list formats of
srwlpy.PropagElecField's intList, and on the GPU the drop-in's extractions against the fixtures."""
import json
import os
import sys
from array import array

import numpy as np
import pytest

from srw_b200 import srwlpy
from srw_b200.srwlib import SRWLRadMesh
from tests.golden_cases import cplx, load, mesh_dict, rel_l2
from tests.helpers import beamline, make_wfr

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), 'oracle'))
import srw_oracle as O  # noqa: E402

D, _ = load()
XINDEX = json.loads(str(D['xint/index']))
WHAT = {0: 0, 4: 2, 5: 3, 6: 6}
TOL_ORACLE = 1e-5        # FP64 oracle vs the FP32 reference (relative L2)
TOL_GPU = 1e-4           # FP32 GPU path vs the FP32 reference


def case_input(c):
    m = D['xint/%s/in/mesh' % c['name']]
    nx, ny = int(m[0]), int(m[1])
    sc = D['xint/%s/in/scal' % c['name']]
    return dict(ex=cplx(D['xint/%s/in/ex' % c['name']], nx, ny), ey=cplx(D['xint/%s/in/ey' % c['name']], nx, ny),
                mesh=mesh_dict(m), Rx=float(sc[0]), Ry=float(sc[1]), dRx=float(sc[2]), dRy=float(sc[3]),
                xc=float(sc[4]), yc=float(sc[5]), momX=np.array(D['xint/%s/in/momx' % c['name']]),
                momY=np.array(D['xint/%s/in/momy' % c['name']]), prop=np.array(D['xint/%s/in/prop' % c['name']]))


def effective(reqs):
    """Negative values of the later requests take the first request's (sroptcnt.cpp:453-460)."""
    out = []
    for i, (el, pol, typ) in enumerate(reqs):
        if i > 0:
            pol = reqs[0][1] if pol < 0 else pol
            typ = reqs[0][2] if typ < 0 else typ
        out.append((el, pol, typ))
    return out


@pytest.mark.parametrize('name', [c['name'] for c in XINDEX])
def test_oracle_extractions_vs_reference(name):
    c = next(c for c in XINDEX if c['name'] == name)
    i = case_input(c)
    w = O.Wfr.from_srwl(i['ex'], i['ey'], i['mesh'], i['Rx'], i['Ry'], i['dRx'], i['dRy'], i['xc'], i['yc'], 0,
                        i['momX'], i['momY'], propM=i['prop'])
    reqs = effective(c['reqs'])
    seen = []

    def after(k, w):
        for j, (el, pol, typ) in enumerate(reqs):
            if el - 1 == k:
                m = w.out_mesh()
                seen.append(j)
                ref_m = D['xint/%s/%d/mesh' % (name, j)]
                assert np.array_equal([m['nx'], m['ny'], m['xStart'], m['xFin'], m['yStart'], m['yFin']], ref_m[:6])
                I = O.calc_int_from_elec_field(w.ex, w.ey, pol, typ)
                assert rel_l2(I, D['xint/%s/%d/I' % (name, j)]) < TOL_ORACLE, (j, el, pol, typ)
    O.propagate(w, [tuple(e) for e in c['elements']], c['props'], after=after)
    assert sorted(seen) == list(range(len(reqs)))


def test_int_list_formats():
    """ParseSructSRWLPropIntDef / UpdatePyPropInt (srwlpy.cpp:2784, 3809): the flat format gets each
    array appended to its request; the column format gets a mesh list and an array list (one value
    for all requests is repeated, the later ones inheriting), or the single array."""
    m0, m1 = SRWLRadMesh(), SRWLRadMesh()
    flat = [[1, 6, 0, 3, 0, m0], [2, -1, 5, 3, 0, m1]]
    reqs, meshes, isflat = srwlpy._parse_int_list(flat)
    assert isflat and reqs == [[1, 6, 0, 3, 0], [2, -1, 5, 3, 0]] and meshes == [m0, m1]
    cols = [[1, 3], 6, 0, 3, 0, m0]
    reqs, meshes, isflat = srwlpy._parse_int_list(cols)
    assert not isflat and reqs == [[1, 6, 0, 3, 0], [3, -1, -1, -1, -1]] and meshes == [m0, None]

    class CM(object):      # a C mesh as the library leaves it
        def __init__(self, nx):
            self.eStart = self.eFin = 1000.
            self.xStart, self.xFin, self.yStart, self.yFin = -1., 1., -2., 2.
            self.ne, self.nx, self.ny = 1, nx, nx + 1
    a0, a1 = array('f', [1.]), array('f', [2.])
    srwlpy._update_int_list(flat, True, [m0, m1], [CM(4), CM(8)], [a0, a1])
    assert flat[0][6] is a0 and flat[1][6] is a1 and m0.nx == 4 and m1.ny == 9
    srwlpy._update_int_list(cols, False, [m0, None], [CM(5), CM(6)], [a0, a1])
    assert cols[5][0] is m0 and cols[5][1] is not m0 and cols[5][1].nx == 6 and cols[6] == [a0, a1]
    single = [2, 6, 0, 3, 0, SRWLRadMesh()]
    srwlpy._update_int_list(single, False, [single[5]], [CM(7)], [a0])
    assert single[6] is a0 and single[5].nx == 7


@pytest.mark.gpu
@pytest.mark.parametrize('name', [c['name'] for c in XINDEX])
def test_gpu_extractions_vs_reference(name):
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    c = next(c for c in XINDEX if c['name'] == name)
    i = case_input(c)
    w = make_wfr(i['ex'], i['ey'], i['mesh'], Rx=i['Rx'], Ry=i['Ry'], dRx=i['dRx'], dRy=i['dRy'], xc=i['xc'],
                 yc=i['yc'], momX=i['momX'], momY=i['momY'], propM=i['prop'])
    intList = [[el, pol, typ, 3, 0, SRWLRadMesh(i['mesh']['eStart'], i['mesh']['eStart'], 1)]
               for el, pol, typ in c['reqs']]
    srwlpy.PropagElecField(w, beamline(c['elements'], c['props']), intList)
    for j, it in enumerate(intList):
        m = it[5]
        ref_m = D['xint/%s/%d/mesh' % (name, j)]
        assert np.array_equal([m.nx, m.ny, m.xStart, m.xFin, m.yStart, m.yFin], ref_m[:6]), j
        assert (m.ne, m.eStart) == (1, ref_m[6])
        assert rel_l2(np.asarray(it[6], np.float64), D['xint/%s/%d/I' % (name, j)]) < TOL_GPU, j
    out = D['xint/%s/out/ex' % name]
    assert rel_l2(np.asarray(w.arEx, np.float64), out) < TOL_GPU


@pytest.mark.gpu
def test_gpu_phase_and_column_format():
    """The phase (type 4, FP64 array) and the column list format, against the oracle's state after
    the element (where the intensity is above 1e-3 of its peak)."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    c = next(c for c in XINDEX if c['name'] == 'x_c0')
    i = case_input(c)
    w = make_wfr(i['ex'], i['ey'], i['mesh'], Rx=i['Rx'], Ry=i['Ry'], dRx=i['dRx'], dRy=i['dRy'])
    mesh = SRWLRadMesh(i['mesh']['eStart'], i['mesh']['eStart'], 1)
    intList = [[1, 3], 6, 4, 3, 0, mesh]         # phase after the first drift and after the lens
    srwlpy.PropagElecField(w, beamline(c['elements'], c['props']), intList)
    assert isinstance(intList[6], list) and len(intList[6]) == 2 and intList[6][0].typecode == 'd'
    ow = O.Wfr.from_srwl(i['ex'], i['ey'], i['mesh'], i['Rx'], i['Ry'], i['dRx'], i['dRy'], 0., 0., 0, None, None)
    states = {}
    O.propagate(ow, [tuple(e) for e in c['elements']], c['props'],
                after=lambda k, s: states.setdefault(k, (s.ex.copy(), s.ey.copy())))
    for j, k in enumerate((0, 2)):
        ex, ey = states[k]
        I = np.abs(ex) ** 2 + np.abs(ey) ** 2
        sel = (I > 1e-3 * I.max()).ravel()
        ph = np.asarray(intList[6][j], np.float64)
        ref = O.calc_int_from_elec_field(ex, ey, 6, 4)
        d = np.angle(np.exp(1j * (ph[sel] - ref[sel])))
        assert np.max(np.abs(d)) < 2e-3, (j, np.max(np.abs(d)))
        assert intList[5][j].nx == ex.shape[1]


@pytest.mark.gpu
def test_gpu_unsupported_extraction_refused():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    c = next(c for c in XINDEX if c['name'] == 'x_c0')
    i = case_input(c)
    w = make_wfr(i['ex'], i['ey'], i['mesh'])
    with pytest.raises(RuntimeError, match='dep 3'):
        srwlpy.PropagElecField(w, beamline(c['elements'], c['props']), [[1, 6, 0, 1, 0, SRWLRadMesh()]])


@pytest.mark.gpu
def test_gpu_extractions_across_stages():
    """A chain planned in stages (a pp[3]=1 drift after an aperture that recomputes the moments): the
    extractions of every stage reach the caller, against the oracle's state after each element."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from tests.golden_cases import case_io
    name = 'quad1_clip'
    c = next(c for c in load()[1] if c['name'] == name)
    i, o = case_io(D, name)
    w = make_wfr(i['ex'], i['ey'], i['mesh'], Rx=i['Rx'], Ry=i['Ry'], dRx=i['dRx'], dRy=i['dRy'], xc=i['xc'],
                 yc=i['yc'], momX=i['momX'], momY=i['momY'], propM=i['prop'])
    n = len(c['elements'])
    intList = [[k + 1, 6, 0, 3, 0, SRWLRadMesh(i['mesh']['eStart'], i['mesh']['eStart'], 1)] for k in range(n)]
    srwlpy.PropagElecField(w, beamline(c['elements'], c['props']), intList)
    ow = O.Wfr.from_srwl(i['ex'], i['ey'], i['mesh'], i['Rx'], i['Ry'], i['dRx'], i['dRy'], i['xc'], i['yc'], 0,
                         i['momX'], i['momY'], propM=i['prop'])
    states = {}
    O.propagate(ow, [tuple(e) for e in c['elements']], c['props'],
                after=lambda k, s: states.setdefault(k, (s.ex.copy(), s.ey.copy(), s.out_mesh())))
    for k in range(n):
        ex, ey, m = states[k]
        it = intList[k]
        assert (it[5].nx, it[5].ny) == (m['nx'], m['ny'])
        np.testing.assert_allclose([it[5].xStart, it[5].xFin, it[5].yStart, it[5].yFin],
                                   [m['xStart'], m['xFin'], m['yStart'], m['yFin']], rtol=1e-8)
        I = np.abs(ex) ** 2 + np.abs(ey) ** 2
        assert rel_l2(np.asarray(it[6], np.float64), I.ravel()) < TOL_GPU, k
    assert rel_l2(np.asarray(w.arEx, np.float64), D[name + '/out/ex']) < TOL_GPU
