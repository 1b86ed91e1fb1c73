"""Gaussian beam field generation (srwlCalcElecFieldGaussian, one photon energy, no automatic
sampling): the oracle's restatement against the reference's own outputs (golden: waist at the
observation plane, offsets / angles / Hermite modes, every polarisation, field units, spectral
detuning), and on the GPU the drop-in against the same outputs."""
import json
import os
import sys

import numpy as np
import pytest

from tests.golden_cases import GOLDEN, moment_err, rel_l2

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), 'oracle'))
import srw_oracle as O  # noqa: E402  (the checker)

D = np.load(GOLDEN)
CASES = json.loads(str(D['gauss/index']))
FIELD_TOL = 1e-6      # relative L2: the reference rounds the field once more (quadratic-phase removal
                      # and re-addition around its moment computation); FP64 math rounded to FP32
MOM_TOL = 1e-5        # each moment relative to its scale
PROP_IN = [0.] * 16 + [1e-4, 2e-6, -3e-4, 4e-6]


def ref(name, m):
    g = lambda k: D['gauss/%s/%s' % (name, k)]  # noqa: E731
    ex, ey = g('ex'), g('ey')
    return ((ex[0::2] + 1j * ex[1::2]).reshape(m['ny'], m['nx']), (ey[0::2] + 1j * ey[1::2]).reshape(m['ny'], m['nx']),
            g('scal'), g('momx'), g('momy'), g('prop'))


def check(name, m, ex, ey, scal, momx, momy, prop):
    rx, ry, rs, rmx, rmy, rp = ref(name, m)
    assert rel_l2(ex, rx) < FIELD_TOL and rel_l2(ey, ry) < FIELD_TOL, name
    assert list(scal) == list(rs[:6]), name
    assert moment_err(momx, rmx) < MOM_TOL, name
    if np.any(rmy):
        assert moment_err(momy, rmy) < MOM_TOL, name
    else:
        assert not np.any(momy)
    np.testing.assert_array_equal(prop, rp)


def test_oracle_matches_reference():
    assert len(CASES) == 6
    for c in CASES:
        w, p = O.calc_elec_field_gaussian(c['mesh'], c['beam'], c['unit'])
        check(c['name'], c['mesh'], w.ex, w.ey, [w.RobsX, w.RobsZ, w.RobsXAbsErr, w.RobsZAbsErr, w.xc, w.zc],
              w.momX, w.momZ, np.concatenate([p, PROP_IN[16:]]))


@pytest.mark.gpu
def test_gpu_matches_reference():
    torch = pytest.importorskip('torch')
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from array import array
    from srw_b200 import srwlpy as srwl
    from srw_b200.srwlib import SRWLGsnBm, SRWLWfr
    for c in CASES:
        m = c['mesh']
        gb = SRWLGsnBm()
        for k, v in c['beam'].items():
            setattr(gb, k, v)
        w = SRWLWfr()
        w.allocate(1, m['nx'], m['ny'])
        for k in ('xStart', 'xFin', 'yStart', 'yFin', 'eStart', 'eFin', 'zStart'):
            setattr(w.mesh, k, m[k])
        w.unitElFld = c['unit']
        w.arElecPropMatr = array('d', PROP_IN)
        srwl.CalcElecFieldGaussian(w, gb, [0])
        ex = np.array(w.arEx, np.float32)
        ey = np.array(w.arEy, np.float32)
        ex = (ex[0::2] + 1j * ex[1::2]).reshape(m['ny'], m['nx'])
        ey = (ey[0::2] + 1j * ey[1::2]).reshape(m['ny'], m['nx'])
        check(c['name'], m, ex, ey, [w.Rx, w.Ry, w.dRx, w.dRy, w.xc, w.yc], np.array(w.arMomX), np.array(w.arMomY),
              np.array(w.arElecPropMatr))
