"""Generic transmission element (SRWLOptT, cpp/src/core/sroptgtr.h): the Python structure follows the
reference's constructor, the planner lowers it into a point-wise table lookup of the coordinate-side
pass, and on the GPU it agrees with the FP64 oracle on tables of any grid (finer or coarser than the
wavefront, narrower than it with zero or boundary values outside, off centre), and an identity table
leaves the field bit-for-bit unchanged at full size."""
import numpy as np
import pytest

from srw_b200.plan import Plan
from srw_b200.srwlib import SRWLOptC, SRWLOptD, SRWLOptT
from tests.helpers import PP, beamline, fields, gaussian, make_wfr, oracle_run, rel_l2

TOL = 1e-4           # relative L2, FP32 path vs FP64 oracle


def table(nx, ny, rx, ry, x, y, F, ripple, seed, amp=0.3):
    """(T, OPD) pairs over [ny][nx]: a focusing path -(r^2)/(2F) plus a seeded ripple, T falling off
    towards the edges."""
    g = np.random.default_rng(seed)
    X, Y = np.meshgrid(np.linspace(-0.5 * rx, 0.5 * rx, nx), np.linspace(-0.5 * ry, 0.5 * ry, ny))
    kx, ky = (2. * np.pi / rx) * g.uniform(1., 4.), (2. * np.pi / ry) * g.uniform(1., 4.)
    out = np.empty((ny, nx, 2))
    out[..., 0] = 1. - amp * (X * X / (0.25 * rx * rx) + Y * Y / (0.25 * ry * ry)) + 0.02 * g.standard_normal(X.shape)
    out[..., 1] = -(X * X + Y * Y) / (2. * F) + ripple * np.sin(kx * X) * np.cos(ky * Y)
    return out.ravel()


def test_structure_follows_the_reference_constructor():
    t = SRWLOptT(5, 4, 2e-3, 1e-3, None, 1, 3., 4., 0.1e-3, -0.2e-3)
    assert len(t.arTr) == 2 * 5 * 4 and t.mesh.nx == 5 and t.mesh.ny == 4 and t.mesh.ne == 1
    assert (t.mesh.xStart, t.mesh.xFin) == (0.1e-3 - 1e-3, 0.1e-3 + 1e-3)
    assert (t.mesh.yStart, t.mesh.yFin) == (-0.2e-3 - 0.5e-3, -0.2e-3 + 0.5e-3)
    assert (t.extTr, t.Fx, t.Fy) == (1, 3., 4.)
    a = np.ones(2 * 3 * 3)
    assert SRWLOptT(3, 3, 1e-3, 1e-3, a).arTr is a       # a table of the right length is kept


def test_plan_lowers_the_table_into_the_first_pass():
    ex, ey, mesh = gaussian(128, E=10000., sig=20e-6, r=0.5e-3, R=30.)
    w = make_wfr(ex, ey, mesh, Rx=30., Ry=30., dRx=0.3, dRy=0.3)
    tr = ('transmission', table(33, 29, 0.2e-3, 0.2e-3, 0., 0., 200., 2e-11, 0), 33, 29, 0.2e-3, 0.2e-3, 0., 0., 0,
          200., 200.)
    p = Plan(w, beamline([tr, ('drift', 5., 0)], [PP(), PP()]))
    q = Plan(w, beamline([('drift', 5., 0)], [PP()]))
    # the table rides on the drift's first line pass: no extra pass, the table bytes appended
    assert p.n_kernels == q.n_kernels
    # a table that is too short for its mesh is refused by the marshalling
    bad = SRWLOptT(33, 29, 0.2e-3, 0.2e-3, np.ones(2 * 33 * 29))
    bad.arTr = np.ones(10)
    with pytest.raises(RuntimeError, match='Transmission'):
        Plan(w, SRWLOptC([bad, SRWLOptD(1.)], [PP(), PP()]))


CASES = {
    # finer than the wavefront, narrower than the beam (zero outside), off centre, then a drift
    'fine_narrow_offc': (256, [('transmission', table(301, 257, 0.12e-3, 0.1e-3, 0.01e-3, -0.005e-3, 200., 2e-11, 3),
                                301, 257, 0.12e-3, 0.1e-3, 0.01e-3, -0.005e-3, 0, 200., 200.), ('drift', 10., 0)],
                         [PP(), PP()]),
    # coarser, boundary values outside, before a drift to the waist
    'coarse_ext_towaist': (256, [('transmission', table(23, 31, 0.1e-3, 0.12e-3, 0., 0., 200., 2e-11, 4), 23, 31,
                                  0.1e-3, 0.12e-3, 0., 0., 1, 200., 200.), ('drift', 12., 0)], [PP(), PP(4)]),
    # after a drift (the field is brought back to coordinates first), then a resize and a lens
    'after_drift': (192, [('drift', 3., 0), ('transmission', table(64, 64, 0.3e-3, 0.3e-3, 0., 0., 300., 1e-11, 5), 64,
                                             64, 0.3e-3, 0.3e-3, 0., 0., 0, 300., 300.),
                          ('lens', 20., 20., 0., 0.), ('drift', 5., 0)],
                    [PP(), PP(0, 1., 1.5, 1., 1.5), PP(), PP()]),
}


@pytest.mark.gpu
@pytest.mark.parametrize('name', sorted(CASES))
def test_transmission_vs_oracle(name):
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from srw_b200 import srwlpy as srwl
    n, els, pps = CASES[name]
    ex, ey, mesh = gaussian(n, E=10000., sig=20e-6, r=0.5e-3, R=30.)
    ey = 0.3j * ex
    sc = dict(Rx=30., Ry=30., dRx=0.3, dRy=0.3)
    w = make_wfr(ex, ey, mesh, **sc)
    srwl.PropagElecField(w, beamline(els, pps))
    o = oracle_run(ex, ey, mesh, els, pps, **sc)
    m = o.out_mesh()
    assert (w.mesh.nx, w.mesh.ny, w.mesh.xStart, w.mesh.xFin) == (m['nx'], m['ny'], m['xStart'], m['xFin'])
    assert [w.Rx, w.Ry, w.xc, w.yc] == [o.RobsX, o.RobsZ, o.xc, o.zc]
    gx, gy = fields(w)
    assert rel_l2(gx, o.ex) < TOL and rel_l2(gy, o.ey) < TOL
    np.testing.assert_allclose(np.array(w.arMomX)[:11], o.momX[:11], rtol=1e-12)


@pytest.mark.gpu
def test_identity_table_leaves_the_field_unchanged_at_full_size():
    """T = 1, OPD = 0 over a mesh wider than the wavefront: the field after (transmission, drift) is
    bit-identical to the field after the drift alone (2048^2)."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from srw_b200 import srwlpy as srwl
    ex, ey, mesh = gaussian(2048, E=10000., sig=20e-6, r=0.5e-3, R=30.)
    ident = np.zeros(2 * 17 * 17)
    ident[0::2] = 1.
    outs = []
    for els, pps in (([('drift', 10., 0)], [PP()]),
                     ([('transmission', ident, 17, 17, 2e-3, 2e-3, 0., 0., 0, 1e23, 1e23), ('drift', 10., 0)],
                      [PP(), PP()])):
        w = make_wfr(ex, ey, mesh, Rx=30., Ry=30., dRx=0.3, dRy=0.3)
        srwl.PropagElecField(w, beamline(els, pps))
        outs.append((np.array(w.arEx, np.float32), w.mesh.nx, w.mesh.xStart, w.Rx))
    assert outs[0][1:] == outs[1][1:]
    assert np.array_equal(outs[0][0], outs[1][0])
