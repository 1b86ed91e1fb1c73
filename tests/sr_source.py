"""The undulator source of the headline beamline, computed by the reference SRW itself (its srwlpy
extension built from source by oracle/Makefile): test infrastructure for full-size parity runs on
the reference's own field.

srwlpy reads its arguments by attribute name and recognises magnetic-field objects by class name
(cpp/src/clients/python/srwlpy.cpp:1195-1280, 1620-1670), so the small classes below carry the
reference's names and attributes (env/python/srwpy/srwlib.py: SRWLMagFldH :306, SRWLMagFldU :325,
SRWLMagFldC :410); the wavefront and particle beam are srw_b200.srwlib's.
"""
from array import array

import numpy as np

from srw_b200 import srwlib as S


class SRWLMagFldH(object):
    """One harmonic of an undulator field: number, plane ('v' or 'h'), peak field [T], phase,
    symmetry (1 symmetric, -1 antisymmetric), coefficient."""

    def __init__(self, _n=1, _h_or_v='v', _B=0., _ph=0., _s=1, _a=1.):
        self.n, self.h_or_v, self.B, self.ph, self.s, self.a = _n, _h_or_v, _B, _ph, _s, _a


class SRWLMagFldU(object):
    """Periodic (undulator) field: harmonics, period [m], number of periods."""

    def __init__(self, _arHarm=None, _per=0.02, _nPer=10):
        self.arHarm, self.per, self.nPer = list(_arHarm or []), _per, _nPer


class SRWLMagFldC(object):
    """Container of magnetic fields with their centre positions [m]."""

    def __init__(self, _arMagFld, _arXc, _arYc, _arZc):
        self.arMagFld = list(_arMagFld)
        self.arXc, self.arYc, self.arZc = _arXc, _arYc, _arZc


def undulator_wfr(srwlpy, n, r=1.5e-3, z=20., npTraj=20000):
    """First-harmonic field of a planar undulator (3 GeV, 0.5 A filament beam, 20 mm x 100 periods,
    K = 1.5, By = K / (0.0934 per[mm])) at distance z on an n x n mesh over +-r, computed with the
    reference's CalcElecFieldSR (precPar = [1, 0.01, 0, 0, npTraj, 1, 0]).  Returns the srw_b200
    SRWLWfr (float32 fields, R, dR and moments as the reference leaves them)."""
    per, nper, K = 0.02, 100, 1.5
    By = K / (0.0934 * per * 1000.)
    mag = SRWLMagFldC([SRWLMagFldU([SRWLMagFldH(1, 'v', By, 0, 1, 1)], per, nper)], array('d', [0]), array('d', [0]),
                      array('d', [0]))
    eb = S.SRWLPartBeam()
    eb.Iavg = 0.5
    eb.partStatMom1.x = eb.partStatMom1.y = eb.partStatMom1.xp = eb.partStatMom1.yp = 0.
    eb.partStatMom1.z = -0.5 * per * (nper + 4)
    eb.partStatMom1.gamma = 3. / 0.51099890221e-03
    lam1 = per / (2. * eb.partStatMom1.gamma ** 2) * (1. + K * K / 2.)
    E1 = 1.239842e-06 / lam1
    w = S.SRWLWfr()
    w.allocate(1, n, n)
    w.arEx = np.zeros(2 * n * n, np.float32)
    w.arEy = np.zeros(2 * n * n, np.float32)
    m = w.mesh
    m.zStart, m.eStart, m.eFin = z, E1, E1
    m.xStart, m.xFin, m.yStart, m.yFin = -r, r, -r, r
    w.partBeam = eb
    srwlpy.CalcElecFieldSR(w, 0, mag, [1, 0.01, 0., 0., npTraj, 1, 0])
    return w
