"""GPU parity: the CUDA path (through the srwlpy-compatible drop-in, i.e. the C-ABI) against the
reference SRW's outputs (golden fixtures, and the reference built from source when it is
present) and the FP64 oracle.  Bar: meshes and wavefront scalars bit-exact; complex field and
intensity within relative L2 1e-4 (FP32 path vs FP64 oracle / FP32 reference)."""
import os
import sys

import numpy as np
import pytest

torch = pytest.importorskip('torch')
pytestmark = pytest.mark.gpu

from srw_b200 import srwlpy as srwl  # noqa: E402
from srw_b200.plan import Plan  # noqa: E402
from tests.golden_cases import MOMENT_RECOMPUTED, STAGED, case_io, load, mesh_close, moment_err  # noqa: E402
from tests.helpers import (C0, C0PP, C1, C1PP, C2, C2PP, PP, beamline, fields, gaussian, make_wfr,  # noqa: E402
                           mesh_tuple, oracle_run, rel_l2)

TOL = 1e-4           # relative L2, field and intensity
D, INDEX = load()
REF_DIR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), 'oracle', '_ref')


def need_gpu():
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')


def run_gpu(ex, ey, mesh, elements, props, **sc):
    w = make_wfr(ex, ey, mesh, **sc)
    srwl.PropagElecField(w, beamline(elements, props))
    return w


@pytest.mark.parametrize('name', [c['name'] for c in INDEX])
def test_golden_case(name):
    need_gpu()
    c = next(c for c in INDEX if c['name'] == name)
    i, o = case_io(D, name)
    w = run_gpu(i['ex'], i['ey'], i['mesh'], c['elements'], c['props'], Rx=i['Rx'], Ry=i['Ry'], dRx=i['dRx'],
                dRy=i['dRy'], xc=i['xc'], yc=i['yc'], momX=i['momX'], momY=i['momY'], propM=i['prop'])
    assert mesh_close(mesh_tuple(w), o['mesh_raw'], name in STAGED)
    np.testing.assert_allclose(np.array(w.arElecPropMatr), o['prop'], rtol=1e-14, atol=1e-300)
    scal = [w.Rx, w.Ry, w.dRx, w.dRy, w.xc, w.yc]
    ref = [o['Rx'], o['Ry'], o['dRx'], o['dRy'], o['xc'], o['yc']]
    if name in STAGED:      # planned on moments measured from the FP32 field
        np.testing.assert_allclose(scal, ref, rtol=1e-8, atol=1e-20)
    else:
        assert scal == ref
    ex, ey = fields(w)
    assert rel_l2(ex, o['ex']) < TOL
    if np.linalg.norm(o['ey']) > 0:
        assert rel_l2(ey, o['ey']) < TOL
    else:
        assert np.linalg.norm(ey) == 0.
    assert rel_l2(np.abs(ex) ** 2 + np.abs(ey) ** 2, np.abs(o['ex']) ** 2 + np.abs(o['ey']) ** 2) < TOL
    if name not in MOMENT_RECOMPUTED:
        np.testing.assert_allclose(np.array(w.arMomX), o['momX'], rtol=1e-12)
        np.testing.assert_allclose(np.array(w.arMomY), o['momY'], rtol=1e-12)
    else:       # recomputed from the FP32 field: each moment to 1e-4 of its scale
        assert moment_err(np.array(w.arMomX), o['momX']) < TOL
        assert moment_err(np.array(w.arMomY), o['momY']) < TOL


def full_case(which):
    if which == 'c0':
        ex, ey, mesh = gaussian(512, E=1000., sig=50e-6, r=1e-3)
        return ex, ey, mesh, C0, C0PP, {}
    if which == 'c1':
        # curved 2 keV beam 20 m from its source, 1024^2 over +-1.5 mm (undulator-like envelope)
        ex, ey, mesh = gaussian(1024, E=2012., sig=0.35e-3, r=1.5e-3, R=20.)
        ey = 0.05j * ex
        return ex, ey, mesh, C1, C1PP, dict(Rx=20., Ry=20., dRx=0.2, dRy=0.2)
    ex, ey, mesh = gaussian(4096, E=10000., sig=20e-6, r=1e-3, R=30.)
    if which == 'c2q1':
        # the pp[3]=1 variant: radius estimate from the rms divergence; the input has no moments, so
        # the first drift measures them on the 4096^2 field (a stage boundary)
        return ex, ey, mesh, C2, [PP(1), PP(), PP(1)], dict(Rx=30., Ry=30., dRx=0.3, dRy=0.3)
    return ex, ey, mesh, C2, C2PP, dict(Rx=30., Ry=30., dRx=0.3, dRy=0.3)


def phase_err(a, b, rel=1e-3):
    """Intensity-weighted RMS of the phase difference arg(a conj(b)) [rad] where |b|^2 exceeds `rel`
    of its maximum."""
    I = np.abs(b) ** 2
    sel = I > rel * I.max()
    d = np.angle(a[sel] * np.conj(b[sel]))
    return float(np.sqrt(np.sum(I[sel] * d * d) / np.sum(I[sel])))


def report(**kv):
    """Appends the figures of a test to $SRWG_TEST_REPORT (JSON lines) when that is set."""
    path = os.environ.get('SRWG_TEST_REPORT')
    if path:
        import json
        with open(path, 'a') as f:
            f.write(json.dumps(kv) + '\n')


@pytest.mark.parametrize('which', ['c0', 'c1', 'c2', 'c2q1'])
def test_full_size_vs_fp64_oracle(which):
    need_gpu()
    ex, ey, mesh, el, pp, sc = full_case(which)
    w = run_gpu(ex, ey, mesh, el, pp, **sc)
    o = oracle_run(ex, ey, mesh, el, pp, **sc)
    m = o.out_mesh()
    assert mesh_close(mesh_tuple(w), np.array([m['nx'], m['ny'], m['xStart'], m['xFin'], m['yStart'], m['yFin']]),
                      which == 'c2q1')
    if which == 'c2q1':
        assert moment_err(np.array(w.arMomX), o.momX) < TOL
    gx, gy = fields(w)
    e_field = rel_l2(gx, o.ex)
    I_g = np.abs(gx) ** 2 + np.abs(gy) ** 2
    I_o = np.abs(o.ex) ** 2 + np.abs(o.ey) ** 2
    e_int = rel_l2(I_g, I_o)
    # phase of Ex against the FP64 oracle (intensity-weighted RMS where the intensity is above 1e-3 of
    # its maximum): 1e-4 rad, the field bar
    e_ph = phase_err(gx, o.ex)
    report(test='full_vs_fp64_oracle', case=which, grid=[int(w.mesh.nx), int(w.mesh.ny)], field_rel_l2=e_field,
           intensity_rel_l2=e_int, phase_rms_rad=e_ph)
    assert e_field < TOL
    assert e_int < TOL
    assert e_ph < TOL


def _reference():
    if not os.path.exists(os.path.join(REF_DIR, 'srwlpy.so')):
        pytest.skip('reference build (oracle/_ref) not present')
    if REF_DIR not in sys.path:
        sys.path.insert(0, REF_DIR)
    import srwlpy as ref
    return ref


def _copy_wfr(w):
    ex, ey = fields(w)
    m = w.mesh
    mesh = dict(xStart=m.xStart, xFin=m.xFin, yStart=m.yStart, yFin=m.yFin, eStart=m.eStart, eFin=m.eFin,
                zStart=m.zStart)
    return make_wfr(ex, ey, mesh, Rx=w.Rx, Ry=w.Ry, dRx=w.dRx, dRy=w.dRy, xc=w.xc, yc=w.yc,
                    momX=list(w.arMomX) if w.arMomX is not None else None,
                    momY=list(w.arMomY) if w.arMomY is not None else None)


def _vs_reference(w0, el, pp, name):
    ref = _reference()
    wr, wg = _copy_wfr(w0), _copy_wfr(w0)
    ref.PropagElecField(wr, beamline(el, pp))
    srwl.PropagElecField(wg, beamline(el, pp))
    assert np.array_equal(mesh_tuple(wg), mesh_tuple(wr))
    assert [wg.Rx, wg.Ry, wg.xc, wg.yc] == [wr.Rx, wr.Ry, wr.xc, wr.yc]
    rx, ry = fields(wr)
    gx, gy = fields(wg)
    e_field = rel_l2(gx, rx)
    e_int = rel_l2(np.abs(gx) ** 2 + np.abs(gy) ** 2, np.abs(rx) ** 2 + np.abs(ry) ** 2)
    e_ph = phase_err(gx, rx)
    report(test='full_vs_reference', case=name, grid=[int(wg.mesh.nx), int(wg.mesh.ny)], field_rel_l2=e_field,
           intensity_rel_l2=e_int, phase_rms_rad=e_ph)
    assert e_field < TOL
    assert e_int < TOL
    assert e_ph < TOL
    return wg, wr


def test_full_c1_undulator_field_vs_reference_built_from_source():
    """The headline beamline (1024^2 -> 4096^2) on the reference's own undulator field (its
    CalcElecFieldSR, 20000 trajectory points), against the reference's propagation of it: the field
    carries the source's moments, so the aperture recomputes them from the field as the reference does."""
    need_gpu()
    from tests.sr_source import undulator_wfr
    w0 = undulator_wfr(_reference(), 1024)
    wg, wr = _vs_reference(w0, C1, C1PP, 'c1_undulator')
    assert int(wg.mesh.nx) == 4096
    assert moment_err(np.array(wg.arMomX), np.array(wr.arMomX)) < TOL


def test_full_c2_vs_reference_built_from_source():
    """4096^2 Gaussian with the imposed 30 m radius through the two quadratic-phase drifts and the
    lens, against the reference's propagation of the same field."""
    need_gpu()
    ex, ey, mesh, el, pp, sc = full_case('c2')
    w0 = make_wfr(ex, ey, mesh, **sc)
    _vs_reference(w0, el, pp, 'c2')


def test_full_c0_vs_reference_built_from_source():
    need_gpu()
    if not os.path.exists(os.path.join(REF_DIR, 'srwlpy.so')):
        pytest.skip('reference build (oracle/_ref) not present')
    sys.path.insert(0, REF_DIR)
    import srwlpy as ref
    ex, ey, mesh, el, pp, sc = full_case('c0')
    wr = make_wfr(ex, ey, mesh, **sc)
    ref.PropagElecField(wr, beamline(el, pp))
    wg = run_gpu(ex, ey, mesh, el, pp, **sc)
    assert np.array_equal(mesh_tuple(wg), mesh_tuple(wr))
    rx, ry = fields(wr)
    gx, gy = fields(wg)
    assert rel_l2(gx, rx) < TOL


def test_device_plan_matches_c_abi_and_batch():
    need_gpu()
    ex, ey, mesh, el, pp, sc = full_case('c0')
    w = make_wfr(ex, ey, mesh, **sc)
    p = Plan(w, beamline(el, pp))
    dex = torch.from_numpy(ex.astype(np.complex64)).cuda()
    dey = torch.from_numpy(ey.astype(np.complex64)).cuda()
    ox, oy = p.new_output()
    p.execute(dex, dey, ox, oy)
    torch.cuda.synchronize()
    wg = run_gpu(ex, ey, mesh, el, pp, **sc)
    gx, _ = fields(wg)
    assert np.array_equal(ox.cpu().numpy(), gx.astype(np.complex64))
    bx = torch.stack([dex, 2 * dex, -1j * dex]).contiguous()
    by = torch.stack([dey, dey, dey]).contiguous()
    obx, oby = p.new_output(batch=3)
    p.execute_batch(bx, by, obx, oby)
    torch.cuda.synchronize()
    ref = ox.cpu().numpy()
    out = obx.cpu().numpy()
    assert rel_l2(out[0], ref) < 1e-6
    assert rel_l2(out[1], 2 * ref) < 1e-6           # linearity
    assert rel_l2(out[2], -1j * ref) < 1e-6
    ms = p.execute_timed(dex, dey, ox, oy)
    assert len(ms) == p.n_kernels and all(t > 0 for t in ms)


def test_drift_round_trip_and_energy():
    """Angular-representation drift is unitary: +L then -L returns the field; power is kept."""
    need_gpu()
    ex, ey, mesh = gaussian(1024, E=1000., sig=60e-6, r=1e-3)
    w = run_gpu(ex, ey, mesh, [('drift', 7., 0), ('drift', -7., 0)], [[0, 0, 1., 0, 0, 1., 1., 1., 1.]] * 2)
    gx, _ = fields(w)
    assert rel_l2(gx, ex) < 1e-5
    w1 = run_gpu(ex, ey, mesh, [('drift', 7., 0)], [[0, 0, 1., 0, 0, 1., 1., 1., 1.]])
    g1, _ = fields(w1)
    assert abs(np.sum(np.abs(g1) ** 2) / np.sum(np.abs(ex) ** 2) - 1.) < 1e-5


def test_odd_input_mesh_resize_then_drift_vs_oracle():
    """Odd input mesh (101 x 75): resize to good numbers then angular drift; exercises the scalar
    (non-vectorised) resize path and the general-radix line passes."""
    need_gpu()
    ex, ey, mesh = gaussian(101, E=1500., sig=80e-6, r=1e-3, ny=75, ry=0.8e-3)
    ey = 0.1 * ex
    el = [('aperture', 'c', 'a', 1.2e-3, 1.2e-3, 0.05e-3, 0.), ('drift', 2., 0)]
    pp = [[0, 0, 1., 0, 0, 1.3, 1.7, 1.2, 1.1, 0, 0, 0], [0, 0, 1., 0, 0, 1., 1., 1., 1., 0, 0, 0]]
    w = run_gpu(ex, ey, mesh, el, pp)
    o = oracle_run(ex, ey, mesh, el, pp)
    m = o.out_mesh()
    assert np.array_equal(mesh_tuple(w), np.array([m['nx'], m['ny'], m['xStart'], m['xFin'], m['yStart'], m['yFin']]))
    gx, gy = fields(w)
    assert rel_l2(gx, o.ex) < TOL
    assert rel_l2(gy, o.ey) < TOL
