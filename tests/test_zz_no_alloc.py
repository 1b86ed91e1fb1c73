"""Allocation-free entry point srwgPropagElecFieldStatic, called through the C-ABI.

It serves callers that cannot allocate device memory while they run (memory reserved once at
start-up, or owned by the caller's own allocator): its intermediate fields live in a fixed array
inside the library.  The test checks that it returns the same fields, mesh and scalars as the
allocating entry point (srwgPlanCreate + srwgPlanExecute), moments included, on two calls in a row, alternating
cases so that the second call of a case follows a different propagation in the shared array,
and that a propagation above the array's limit is refused with a clear error.

This file is collected last on purpose: it must pass alone in a fresh process (where its first
call does the per-device set-up) and after every other test."""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip('torch')
pytestmark = pytest.mark.gpu

from srw_b200 import capi  # noqa: E402
from srw_b200.plan import Plan  # noqa: E402
from srw_b200.srwlpy import make_c_optc, make_c_wfr  # noqa: E402
from tests.golden_cases import case_io, load  # noqa: E402
from tests.helpers import C0, C0PP, C1, C1PP, beamline, gaussian, make_wfr, rel_l2  # noqa: E402

TOL = 1e-4           # relative L2 against the allocating entry point, as in the parity tests
ERR_STATIC_LIMIT = 23904
D, INDEX = load()
CASES = ['c0_128', 'c1_96', 'rs_post', 'ob_circ_lens_offc', 'treat_path', 'c0_512']


def need_gpu():
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')


def case(name):
    if name == 'c0_512':
        ex, ey, mesh = gaussian(512, E=1000., sig=50e-6, r=1e-3)
        return make_wfr(ex, ey, mesh), beamline(C0, C0PP)
    c = next(c for c in INDEX if c['name'] == name)
    i, _ = case_io(D, name)
    w = make_wfr(i['ex'], i['ey'], i['mesh'], Rx=i['Rx'], Ry=i['Ry'], dRx=i['dRx'], dRy=i['dRy'], xc=i['xc'],
                 yc=i['yc'], momX=i['momX'], momY=i['momY'])
    return w, beamline(c['elements'], c['props'])


def to_dev(a, ny, nx):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.complex64).reshape(ny, nx)).cuda()


def run_static(w, optC, ex, ey, nx_out, ny_out):
    keep = []
    cw = make_c_wfr(w, keep)
    co = make_c_optc(optC, keep)
    ox = torch.full((ny_out, nx_out), float('nan'), dtype=torch.complex64, device='cuda')
    oy = torch.full((ny_out, nx_out), float('nan'), dtype=torch.complex64, device='cuda')
    res = capi.SRWLWfr()
    moms = (np.zeros(11), np.zeros(11))
    res.arMomX, res.arMomY = moms[0].ctypes.data, moms[1].ctypes.data
    st = torch.cuda.current_stream().cuda_stream
    r = capi.lib().srwgPropagElecFieldStatic(C.byref(cw), C.byref(co), ex.data_ptr(), ey.data_ptr(), ox.data_ptr(),
                                             oy.data_ptr(), ox.numel(), C.c_void_p(st), C.byref(res))
    torch.cuda.synchronize()
    res.moms = moms
    return r, ox, oy, res


def test_static_matches_plan_twice():
    need_gpu()
    ref = {}
    for name in CASES:
        w, optC = case(name)
        p = Plan(w, optC)
        ex = to_dev(w.arEx, p.ny_in, p.nx_in)
        ey = to_dev(w.arEy, p.ny_in, p.nx_in)
        ox, oy = p.new_output()
        p.execute(ex, ey, ox, oy)
        torch.cuda.synchronize()
        ref[name] = (w, optC, ex, ey, p, ox.cpu().numpy(), oy.cpu().numpy())
    for rep in range(2):
        for name in CASES:
            w, optC, ex, ey, p, rx, ry = ref[name]
            r, ox, oy, res = run_static(w, optC, ex, ey, p.nx_out, p.ny_out)
            assert r == 0, capi.err_text(r)
            gx, gy = ox.cpu().numpy(), oy.cpu().numpy()
            assert np.isfinite(gx).all() and np.isfinite(gy).all()
            assert rel_l2(gx, rx) < TOL, (name, rep)
            if np.linalg.norm(ry) > 0:
                assert rel_l2(gy, ry) < TOL, (name, rep)
            else:
                assert np.linalg.norm(gy) == 0.
            m = p.output_mesh()
            assert (res.mesh.nx, res.mesh.ny) == (m['nx'], m['ny'])
            assert [res.mesh.xStart, res.mesh.xFin, res.mesh.yStart, res.mesh.yFin] == \
                [m['xStart'], m['xFin'], m['yStart'], m['yFin']]
            assert [res.Rx, res.Ry, res.dRx, res.dRy, res.xc, res.yc] == \
                [m['Rx'], m['Ry'], m['dRx'], m['dRy'], m['xc'], m['yc']]
            # moments (recomputed from the field for the aperture / obstacle cases)
            mx, my = p.moments()
            np.testing.assert_allclose(res.moms[0], mx, rtol=1e-6, atol=0)
            np.testing.assert_allclose(res.moms[1], my, rtol=1e-6, atol=0)


def test_static_refuses_above_limit():
    need_gpu()
    ex, ey, mesh = gaussian(1024, E=2012., sig=0.35e-3, r=1.5e-3, R=20.)
    w = make_wfr(ex, ey, mesh, Rx=20., Ry=20., dRx=0.2, dRy=0.2)
    optC = beamline(C1, C1PP)                  # grows the mesh to 4096 x 4096
    dx = torch.zeros((1024, 1024), dtype=torch.complex64, device='cuda')
    r, _, _, _ = run_static(w, optC, dx, dx, 16, 16)
    assert r == ERR_STATIC_LIMIT
    assert 'static limit' in capi.err_text(r)


def test_static_refuses_capturing_stream():
    """Each call copies its tables from host memory, so a call on a stream under capture is refused
    before it queues anything (error 23903); the capture stays valid and later calls work."""
    need_gpu()
    w, optC = case('c0_128')
    p = Plan(w, optC)
    ex = to_dev(w.arEx, p.ny_in, p.nx_in)
    ey = to_dev(w.arEy, p.ny_in, p.nx_in)
    ox, oy = p.new_output()
    keep = []
    cw = make_c_wfr(w, keep)
    co = make_c_optc(optC, keep)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        st = torch.cuda.current_stream().cuda_stream
        r = capi.lib().srwgPropagElecFieldStatic(C.byref(cw), C.byref(co), ex.data_ptr(), ey.data_ptr(),
                                                 ox.data_ptr(), oy.data_ptr(), ox.numel(), C.c_void_p(st), None)
    assert r == 23903
    assert 'captured' in capi.err_text(r)
    r2, gx, _, _ = run_static(w, optC, ex, ey, p.nx_out, p.ny_out)
    assert r2 == 0 and np.isfinite(gx.cpu().numpy()).all()
