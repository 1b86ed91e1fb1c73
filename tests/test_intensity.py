"""Intensity extraction (srwlCalcIntFromElecField vs x and y): the oracle's restatement against the
reference's own outputs (golden vectors: every polarisation, intensity / phase / Re E / Im E, and the
averaging and adding modes), and on the GPU the drop-in against the same vectors."""
import json
import os
import sys

import numpy as np
import pytest

from tests.golden_cases import GOLDEN

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), 'oracle'))
import srw_oracle as O  # noqa: E402  (the checker)

D = np.load(GOLDEN)
CASES = json.loads(str(D['int/index']))
M = D['int/mesh']
NX, NY = int(M[0]), int(M[1])
PHASE_TOL = 5e-7      # rad: the phase is FP64 atan rounded to FP32, one FP32 step at pi is 2.4e-7


def fields():
    ex, ey = D['int/ex'], D['int/ey']
    return ((ex[0::2] + 1j * ex[1::2]).reshape(NY, NX).astype(np.complex64),
            (ey[0::2] + 1j * ey[1::2]).reshape(NY, NX).astype(np.complex64))


def prev(c):
    n = NX * NY * (4 if c['pol'] == -5 else 1)
    return np.sin(np.arange(n) * 0.37).astype(np.float64 if c['int_type'] == 4 else np.float32)


def check(got, c):
    ref = D[c['key']]
    if c['int_type'] == 4:
        assert np.max(np.abs(np.asarray(got, np.float64) - ref)) < PHASE_TOL, c
    else:
        assert np.array_equal(np.asarray(got, np.float32), ref), c      # bit-exact (FP32 operation order)


def test_oracle_matches_reference_vectors():
    assert len(CASES) == 99
    ex, ey = fields()
    for c in CASES:
        check(O.calc_int_from_elec_field(ex, ey, c['pol'], c['int_type'], c['meth'], prev(c)), c)


@pytest.mark.gpu
def test_gpu_matches_reference_vectors():
    torch = pytest.importorskip('torch')
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from srw_b200 import srwlpy as srwl
    from srw_b200.srwlib import SRWLWfr
    w = SRWLWfr()
    w.allocate(1, NX, NY)
    w.arEx = np.array(D['int/ex'], np.float32)
    w.arEy = np.array(D['int/ey'], np.float32)
    w.mesh.xStart, w.mesh.xFin, w.mesh.yStart, w.mesh.yFin = (float(v) for v in M[2:6])
    w.mesh.eStart = w.mesh.eFin = float(M[6])
    for c in CASES:
        arI = prev(c).copy()
        srwl.CalcIntFromElecField(arI, w, c['pol'], c['int_type'], 3, w.mesh.eStart, 0., 0., c['meth'])
        check(arI, c)


CUTS = json.loads(str(D['icut/index']))


def mesh():
    return dict(xStart=float(M[2]), xFin=float(M[3]), yStart=float(M[4]), yFin=float(M[5]))


def test_oracle_cuts_match_reference_vectors():
    """Cuts vs x (dep 1) and vs y (dep 2) and single points (dep 0), between nodes, on a node, below
    the mesh start and beyond its end: bit-exact (phase: to the FP32 step)."""
    assert len(CUTS) == 396
    ex, ey = fields()
    for c in CUTS:
        check(O.calc_int_cut(ex, ey, mesh(), c['pol'], c['int_type'], c['dep'], c['x'], c['y']), c)


@pytest.mark.gpu
def test_gpu_cuts_match_reference_vectors():
    torch = pytest.importorskip('torch')
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from srw_b200 import srwlpy as srwl
    from srw_b200.srwlib import SRWLWfr
    w = SRWLWfr()
    w.allocate(1, NX, NY)
    w.arEx = np.array(D['int/ex'], np.float32)
    w.arEy = np.array(D['int/ey'], np.float32)
    w.mesh.xStart, w.mesh.xFin, w.mesh.yStart, w.mesh.yFin = (float(v) for v in M[2:6])
    w.mesh.eStart = w.mesh.eFin = float(M[6])
    for c in CUTS:
        n = {0: 1, 1: NX, 2: NY}[c['dep']] * (4 if c['pol'] == -5 else 1)
        arI = np.zeros(n, np.float64 if c['int_type'] == 4 else np.float32)
        srwl.CalcIntFromElecField(arI, w, c['pol'], c['int_type'], c['dep'], w.mesh.eStart, c['x'], c['y'])
        check(arI, c)
