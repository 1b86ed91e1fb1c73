"""Wavefront and optical-element structures with the attribute names and constructor arguments of
the reference's Python classes (env/python/srwpy/srwlib.py: SRWLRadMesh :804, SRWLWfr :2200,
SRWLOptD :2908, SRWLOptA :2919, SRWLOptL :2938, SRWLOptT :3036, SRWLOptC :4259) for the drift / lens /
aperture / transmission path.  Objects of the reference's own classes work with ``srw_b200.srwlpy`` as well: elements are
recognised by class name, like the reference's C extension does (srwlpy.cpp:2678).

Field arrays are numpy float32 (``array('f')`` buffers of the reference classes are accepted too).
"""
from array import array

import numpy as np


class SRWLParticle(object):
    def __init__(self, _x=0, _y=0, _z=0, _xp=0, _yp=0, _gamma=1, _relE0=1, _nq=-1):
        self.x, self.y, self.z, self.xp, self.yp = _x, _y, _z, _xp, _yp
        self.gamma, self.relE0, self.nq = _gamma, _relE0, _nq


class SRWLPartBeam(object):
    def __init__(self, _Iavg=0, _nPart=0, _partStatMom1=None, _arStatMom2=None):
        self.Iavg, self.nPart = _Iavg, _nPart
        self.partStatMom1 = SRWLParticle() if _partStatMom1 is None else _partStatMom1
        self.arStatMom2 = array('d', [0] * 21) if _arStatMom2 is None else _arStatMom2


class SRWLRadMesh(object):
    def __init__(self, _eStart=0, _eFin=0, _ne=1, _xStart=0, _xFin=0, _nx=1, _yStart=0, _yFin=0, _ny=1, _zStart=0,
                 _nvx=0, _nvy=0, _nvz=1, _hvx=1, _hvy=0, _hvz=0, _arSurf=None):
        self.eStart, self.eFin, self.ne = _eStart, _eFin, _ne
        self.xStart, self.xFin, self.nx = _xStart, _xFin, _nx
        self.yStart, self.yFin, self.ny = _yStart, _yFin, _ny
        self.zStart = _zStart
        self.nvx, self.nvy, self.nvz, self.hvx, self.hvy, self.hvz = _nvx, _nvy, _nvz, _hvx, _hvy, _hvz
        self.arSurf = _arSurf


class SRWLWfr(object):
    """Electric-field wavefront: arEx/arEy are float32 [ny][nx][ne][re, im] (flat)."""

    def __init__(self, _arEx=None, _arEy=None, _typeE='f', _eStart=0, _eFin=0, _ne=0, _xStart=0, _xFin=0, _nx=0,
                 _yStart=0, _yFin=0, _ny=0, _zStart=0, _partBeam=None):
        self.arEx = _arEx
        self.arEy = _arEy
        # arExAux / arEyAux (backups) exist only after an allocation that asked for them
        self.mesh = SRWLRadMesh(_eStart, _eFin, _ne, _xStart, _xFin, _nx, _yStart, _yFin, _ny, _zStart)
        self.numTypeElFld = _typeE
        self.partBeam = SRWLPartBeam() if _partBeam is None else _partBeam
        self.Rx = self.Ry = 0.
        self.dRx = self.dRy = 0.
        self.xc = self.yc = 0.
        self.avgPhotEn = 0.
        self.presCA = 0
        self.presFT = 0
        self.unitElFld = 1
        self.unitElFldAng = 0
        self.arElecPropMatr = array('d', [0] * 20)
        self.arMomX = array('d', [0] * 11 * _ne)
        self.arMomY = array('d', [0] * 11 * _ne)
        self.arWfrAuxData = array('d', [0] * 30)
        if _ne > 0 and _nx > 0 and _ny > 0 and (_arEx is None or _arEy is None):
            self.allocate(_ne, _nx, _ny, 1 if _arEx is None else 0, 1 if _arEy is None else 0, _typeE)

    def allocate(self, _ne, _nx, _ny, _EXNeeded=1, _EYNeeded=1, _typeE='f', _backupNeeded=0):
        """(Re-)allocates the field arrays for an ne x nx x ny mesh (as SRWLWfr.allocate,
        env/python/srwpy/srwlib.py:2285)."""
        nTot = 2 * _ne * _nx * _ny
        nMom = 11 * _ne
        if _EXNeeded:
            if _backupNeeded:
                self.arExAux = self.arEx
            self.arEx = np.zeros(nTot, np.float32)
            if len(self.arMomX) != nMom:
                self.arMomX = array('d', [0] * nMom)
        if _EYNeeded:
            if _backupNeeded:
                self.arEyAux = self.arEy
            self.arEy = np.zeros(nTot, np.float32)
            if len(self.arMomY) != nMom:
                self.arMomY = array('d', [0] * nMom)
        self.numTypeElFld = _typeE
        self.mesh.ne = _ne
        self.mesh.nx = _nx
        self.mesh.ny = _ny

    def field(self, comp='x'):
        """Complex64 view [ny, nx] of arEx ('x') or arEy ('y') (ne == 1)."""
        a = np.frombuffer(self.arEx if comp == 'x' else self.arEy, dtype=np.float32)
        return a.view(np.complex64).reshape(self.mesh.ny, self.mesh.nx)


class SRWLOptD(object):
    def __init__(self, _L=0, _treat=0):
        self.L = _L
        self.treat = _treat


class SRWLOptA(object):
    def __init__(self, _shape='r', _ap_or_ob='a', _Dx=0, _Dy=0, _x=0, _y=0):
        self.shape = _shape
        self.ap_or_ob = _ap_or_ob
        self.Dx, self.Dy, self.x, self.y = _Dx, _Dy, _x, _y


class SRWLOptL(object):
    def __init__(self, _Fx=1e+23, _Fy=1e+23, _x=0, _y=0):
        self.Fx, self.Fy, self.x, self.y = _Fx, _Fy, _x, _y


class SRWLOptT(object):
    """Generic transmission, the reference's SRWLOptT (env/python/srwpy/srwlib.py:3036) with the same
    constructor signature: ``arTr`` holds (amplitude transmission, optical path difference) pairs,
    C-aligned over [ny][nx] (ne == 1), on a mesh of ranges rx, ry centred on (x, y)."""

    def __init__(self, _nx=1, _ny=1, _rx=1e-03, _ry=1e-03, _arTr=None, _extTr=0, _Fx=1e+23, _Fy=1e+23, _x=0, _y=0,
                 _ne=1, _eStart=0, _eFin=0):
        self.arTr = _arTr
        if _arTr is None or (len(_arTr) != _ne * _nx * _ny * 2 and _ne * _nx * _ny > 0):
            self.allocate(_ne, _nx, _ny)
        hx, hy = 0.5 * _rx, 0.5 * _ry
        if not hasattr(self, 'mesh'):
            self.mesh = SRWLRadMesh(_eStart, _eFin, _ne, _x - hx, _x + hx, _nx, _y - hy, _y + hy, _ny)
        else:
            self.mesh.eStart, self.mesh.eFin = _eStart, _eFin
            self.mesh.xStart, self.mesh.xFin = _x - hx, _x + hx
            self.mesh.yStart, self.mesh.yFin = _y - hy, _y + hy
        self.extTr = _extTr
        self.Fx, self.Fy = _Fx, _Fy

    def allocate(self, _ne, _nx, _ny):
        if hasattr(self, 'mesh'):
            self.mesh.ne, self.mesh.nx, self.mesh.ny = _ne, _nx, _ny
        else:
            self.mesh = SRWLRadMesh(0, 0, _ne, 0, 0, _nx, 0, 0, _ny)
        self.arTr = array('d', [0.]) * (2 * _ne * _nx * _ny)


class SRWLOptC(object):
    def __init__(self, _arOpt=None, _arProp=None):
        self.arOpt = [] if _arOpt is None else _arOpt
        self.arProp = [] if _arProp is None else _arProp


class SRWLGsnBm(object):
    """(Coherent) Gaussian beam at its waist, the reference's SRWLGsnBm (env/python/srwpy/srwlib.py:741)
    with the same attribute names and defaults."""

    def __init__(self, _x=0, _y=0, _z=0, _xp=0, _yp=0, _avgPhotEn=1, _pulseEn=1, _repRate=1, _polar=1, _sigX=10e-06,
                 _sigY=10e-06, _sigT=1e-15, _mx=0, _my=0):
        self.x, self.y, self.z, self.xp, self.yp = _x, _y, _z, _xp, _yp
        self.avgPhotEn, self.pulseEn, self.repRate, self.polar = _avgPhotEn, _pulseEn, _repRate, _polar
        self.sigX, self.sigY, self.sigT, self.mx, self.my = _sigX, _sigY, _sigT, _mx, _my
