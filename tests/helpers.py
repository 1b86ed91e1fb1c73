"""Test helpers: SRWL objects from golden cases, analytic Gaussian inputs, comparisons."""
import os
import sys
from array import array

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(REPO, 'oracle'))
import srw_oracle as O  # noqa: E402  (the checker)

from srw_b200.srwlib import SRWLOptA, SRWLOptC, SRWLOptD, SRWLOptL, SRWLOptT, SRWLWfr  # noqa: E402


def make_wfr(ex, ey, mesh, Rx=0., Ry=0., dRx=0., dRy=0., xc=0., yc=0., momX=None, momY=None, presCA=0, propM=None):
    ny, nx = ex.shape
    w = SRWLWfr()
    w.allocate(1, nx, ny)
    a = np.empty(2 * nx * ny, np.float32)
    a[0::2] = ex.real.ravel(); a[1::2] = ex.imag.ravel()
    w.arEx = a
    b = np.empty(2 * nx * ny, np.float32)
    b[0::2] = ey.real.ravel(); b[1::2] = ey.imag.ravel()
    w.arEy = b
    for k in ('xStart', 'xFin', 'yStart', 'yFin', 'eStart', 'eFin', 'zStart'):
        setattr(w.mesh, k, float(mesh[k]))
    w.mesh.ne, w.mesh.nx, w.mesh.ny = 1, nx, ny
    w.Rx, w.Ry, w.dRx, w.dRy, w.xc, w.yc = Rx, Ry, dRx, dRy, xc, yc
    w.presCA = presCA
    if momX is not None:
        w.arMomX = array('d', list(momX))
        w.arMomY = array('d', list(momY))
    if propM is not None:
        w.arElecPropMatr = array('d', list(propM))
    return w


def beamline(elements, props):
    opts = []
    for e in elements:
        if e[0] == 'drift':
            opts.append(SRWLOptD(e[1], e[2]))
        elif e[0] == 'lens':
            opts.append(SRWLOptL(*e[1:]))
        elif e[0] == 'transmission':
            tr, nx, ny, rx, ry, x, y, ext, Fx, Fy = e[1:11]
            ne, e0, e1 = (e[11:14] if len(e) > 11 else (1, 0., 0.))
            opts.append(SRWLOptT(nx, ny, rx, ry, np.ascontiguousarray(tr, np.float64), ext, Fx, Fy, x, y, ne, e0, e1))
        elif e[0] == 'container':
            opts.append(beamline(e[1], e[2]))
        else:
            opts.append(SRWLOptA(*e[1:]))
    return SRWLOptC(opts, [list(p) for p in props])


def fields(w):
    return w.field('x').astype(np.complex128), w.field('y').astype(np.complex128)


def mesh_tuple(w):
    m = w.mesh
    return np.array([m.nx, m.ny, m.xStart, m.xFin, m.yStart, m.yFin])


def gaussian(n, E=1000., sig=50e-6, r=1e-3, R=0., ny=None, ry=None):
    """Waist (or curved, radius R) Gaussian beam on an n x ny mesh, horizontal polarisation."""
    ny = n if ny is None else ny
    ry = r if ry is None else ry
    x = np.linspace(-r, r, n)[None, :]
    y = np.linspace(-ry, ry, ny)[:, None]
    ex = np.exp(-(x * x + y * y) / (4. * sig * sig)).astype(np.complex128) * 1e6
    if R != 0.:
        lam = 1.239842e-06 / E
        ex = ex * np.exp(1j * np.pi * (x * x + y * y) / (lam * R))
    mesh = dict(nx=n, ny=ny, xStart=-r, xFin=r, yStart=-ry, yFin=ry, eStart=E, eFin=E, zStart=0.)
    return ex, np.zeros_like(ex), mesh


def oracle_run(ex, ey, mesh, elements, props, **sc):
    w = O.Wfr.from_srwl(ex, ey, mesh, sc.get('Rx', 0.), sc.get('Ry', 0.), sc.get('dRx', 0.), sc.get('dRy', 0.),
                        sc.get('xc', 0.), sc.get('yc', 0.), sc.get('presCA', 0), sc.get('momX'), sc.get('momY'))
    O.propagate(w, [tuple(e) for e in elements], props)
    return w


def rel_l2(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / nb) if nb > 0 else float(np.linalg.norm(a))


PP = lambda anal=0, pxm=1., pxd=1., pzm=1., pzd=1.: [0, 0, 1., anal, 0, pxm, pxd, pzm, pzd, 0, 0, 0]  # noqa: E731
C0 = [('drift', 10., 0), ('aperture', 'r', 'a', 1e-3, 1e-3, 0., 0.), ('lens', 5., 5., 0., 0.), ('drift', 5., 0)]
C0PP = [PP()] * 4
C1 = [('aperture', 'c', 'a', 0.8e-3, 0.8e-3, 0., 0.), ('lens', 10., 10., 0., 0.), ('drift', 10., 0)]
C1PP = [PP(), PP(0, 2., 2., 2., 2.), PP(4)]
C2 = [('drift', 30., 0), ('lens', 15., 15., 0., 0.), ('drift', 30., 0)]
C2PP = [PP(2), PP(), PP(2)]
