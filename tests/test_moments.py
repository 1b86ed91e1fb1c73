"""Statistical moments recomputed from the field (ComputeRadMoments) where an aperture clips the
beam or an obstacle sits in it: the planner's moment passes and the host replay of the moment
bookkeeping (CPU), and on the GPU the moments of the drop-in, of the device-resident plans and
of batches against the FP64 oracle."""
import numpy as np
import pytest

from srw_b200.plan import Plan
from tests.golden_cases import moment_err
from tests.helpers import O, beamline, gaussian, make_wfr, oracle_run

TOL = 1e-4        # each moment relative to its scale, FP32 GPU path vs FP64 oracle
PP = [0, 0, 1., 0, 0, 1., 1., 1., 1., 0, 0, 0]


def beam(n=192, x0=0.12e-3, y0=-0.05e-3):
    """Curved 3 keV beam, off centre, with a weaker vertical component of another shape."""
    ex, _, mesh = gaussian(n, E=3000., sig=0.15e-3, r=1e-3, R=15.)
    x = np.linspace(-1e-3, 1e-3, n)[None, :]
    y = np.linspace(-1e-3, 1e-3, n)[:, None]
    env = np.exp(-((x - x0) ** 2 + (y - y0) ** 2) / (4. * 0.15e-3 ** 2)) / np.exp(-(x * x + y * y) / (4. * 0.15e-3 ** 2))
    ex = ex * env
    ey = 0.3j * ex * (1. + 0.5 * x / 1e-3) * np.exp(-(y / 0.6e-3) ** 2)
    sc = dict(Rx=15., Ry=15., dRx=0.15, dRy=0.15)
    w = O.Wfr.from_srwl(ex, ey, mesh, sc['Rx'], sc['Ry'], sc['dRx'], sc['dRy'], 0., 0.)
    O.compute_rad_moments(w)                 # input moments as a source calculation leaves them
    sc['momX'], sc['momY'] = list(w.momX), list(w.momZ)
    return ex, ey, mesh, sc


# obstacle (always recomputes), angular drift, aperture (recomputes if 1.7 sigma is outside it:
# decided on the replayed moments), lens, drift
CHAIN = [('aperture', 'r', 'o', 0.2e-3, 0.1e-3, 0.05e-3, 0.),
         ('drift', 0.5, 0),
         ('aperture', 'c', 'a', 1.0e-3, 1.0e-3, 0.1e-3, 0.05e-3),
         ('lens', 8., 8., 0., 0.),
         ('drift', 2.0, 0)]


def test_plan_has_moment_passes():
    ex, ey, mesh, sc = beam(64)
    p = Plan(make_wfr(ex, ey, mesh, **sc), beamline(CHAIN, [PP] * len(CHAIN)))
    kinds = [k[0] for k in p.kernels()]
    assert kinds.count('moments') == 2          # the obstacle's, and the aperture's after it
    # without input moments an aperture never asks (zero rms sizes sit inside any opening)
    sc0 = dict(sc)
    sc0['momX'] = sc0['momY'] = [0.] * 11
    ch = [CHAIN[2], CHAIN[3], CHAIN[4]]
    p0 = Plan(make_wfr(ex, ey, mesh, **sc0), beamline(ch, [PP] * len(ch)))
    assert 'moments' not in [k[0] for k in p0.kernels()]


def test_oracle_chain_recomputes():
    ex, ey, mesh, sc = beam(64)
    w = oracle_run(ex, ey, mesh, CHAIN, [PP] * len(CHAIN), **sc)
    assert w.momX[0] > 0 and w.momZ[0] > 0
    assert abs(w.momZ[0] / w.momX[0] - 0.09) < 0.05      # |Ey|^2 ~ 0.09 |Ex|^2


# ------------------------------------------------------------------------------------------------
# GPU
# ------------------------------------------------------------------------------------------------
def _gpu():
    torch = pytest.importorskip('torch')
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    return torch


@pytest.mark.gpu
@pytest.mark.parametrize('n', [64, 192, 250])
def test_moments_vs_oracle(n):
    _gpu()
    from srw_b200 import srwlpy as srwl
    ex, ey, mesh, sc = beam(n)
    w = make_wfr(ex, ey, mesh, **sc)
    srwl.PropagElecField(w, beamline(CHAIN, [PP] * len(CHAIN)))
    o = oracle_run(ex, ey, mesh, CHAIN, [PP] * len(CHAIN), **sc)
    assert moment_err(np.array(w.arMomX), o.momX) < TOL
    assert moment_err(np.array(w.arMomY), o.momZ) < TOL


@pytest.mark.gpu
def test_plan_batch_moments_match_single_runs():
    torch = _gpu()
    from srw_b200 import srwlpy as srwl
    ex, ey, mesh, sc = beam(128)
    bl = beamline(CHAIN, [PP] * len(CHAIN))
    p = Plan(make_wfr(ex, ey, mesh, **sc), bl)
    # three wavefronts of the same mesh: scaled, shifted by one column, and the beam itself
    fx = [ex * 2., np.roll(ex, 3, axis=1), ex]
    fy = [ey * 2., np.roll(ey, 3, axis=1), ey * 0.]
    xi = torch.tensor(np.stack(fx).astype(np.complex64)).cuda()
    yi = torch.tensor(np.stack(fy).astype(np.complex64)).cuda()
    xo, yo = p.new_output(3)
    p.execute_batch(xi, yi, xo, yo)
    for b in range(3):
        w = make_wfr(fx[b], fy[b], mesh, **sc)
        srwl.PropagElecField(w, bl)
        mx, my = p.moments(b)
        np.testing.assert_allclose(mx, np.array(w.arMomX), rtol=1e-6, atol=0)
        np.testing.assert_allclose(my, np.array(w.arMomY), rtol=1e-6, atol=0)


# two clipping apertures (the second one's recomputation is decided on the device, and with it the
# quadratic-term treatment flags) before a beyond-paraxial drift that uses those flags
BPX_CHAIN = [('aperture', 'r', 'a', 0.3e-3, 0.3e-3, 0.1e-3, 0.),
             ('aperture', 'c', 'a', 0.5e-3, 0.5e-3, 0.1e-3, 0.05e-3),
             ('lens', 8., 8., 0., 0.),
             ('drift', 8., 0)]
BPX_PP = [PP, PP, PP, [0, 0, 1., 5, 0, 1., 1., 1., 1., 0, 0, 0]]


def test_beyond_paraxial_after_device_decision_needs_stages():
    ex, ey, mesh, sc = beam(64)
    with pytest.raises(RuntimeError, match='plans in stages'):
        Plan(make_wfr(ex, ey, mesh, **sc), beamline(BPX_CHAIN, BPX_PP))


@pytest.mark.gpu
def test_beyond_paraxial_staged_vs_oracle():
    _gpu()
    from srw_b200 import srwlpy as srwl
    from tests.helpers import fields, mesh_tuple, rel_l2
    ex, ey, mesh, sc = beam(128)
    w = make_wfr(ex, ey, mesh, **sc)
    srwl.PropagElecField(w, beamline(BPX_CHAIN, BPX_PP))
    o = oracle_run(ex, ey, mesh, BPX_CHAIN, BPX_PP, **sc)
    m = o.out_mesh()
    np.testing.assert_allclose(mesh_tuple(w), [m['nx'], m['ny'], m['xStart'], m['xFin'], m['yStart'], m['yFin']],
                               rtol=1e-12)
    gx, gy = fields(w)
    assert rel_l2(gx, o.ex) < TOL and rel_l2(gy, o.ey) < TOL
    assert moment_err(np.array(w.arMomX), o.momX) < TOL
