"""Generates the golden fixtures in tests/golden/ by running the reference SRW itself.

Run in a container that has the reference sources (--ref, else $SRW_REFERENCE, else /root/reference) and the reference
built by ``make -C oracle`` (oracle/_ref/srwlpy.so, oracle/_ref/nextfft_probe):

    python tests/golden/make_golden.py [--ref /root/reference]

Outputs (committed):
  good_numbers.txt      runs "first last result" of NextCorrectNumberForFFT(n), n <= 300000
  cases.npz             per case: input field + wavefront scalars, beamline, and the reference's
                        output field, mesh, Rx/Ry/dRx/dRy/xc/yc and moments (float32 fields)
The cases are small (<= 128^2 inputs) so the CPU tests finish in seconds.  Nothing in the
product reads this script; the GPU box never runs it.
"""
import argparse
import json
import os
import subprocess
import sys
from array import array

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def load_reference(ref):
    sys.path.insert(0, os.path.join(REPO, 'oracle', '_ref'))
    sys.path.insert(0, os.path.join(ref, 'env', 'python', 'srwpy'))
    import srwlpy  # noqa: F401  (the reference extension built from source)
    import srwlib
    return srwlib


def gaussian_wfr(L, E, sig, nx, ny, xr, yr, z=0.):
    """Gaussian beam at its waist through the reference's CalcElecFieldGaussian, precPar=[0]."""
    gb = L.SRWLGsnBm()
    gb.x = gb.y = 0.; gb.xp = gb.yp = 0.
    gb.avgPhotEn = E; gb.pulseEn = 0.001; gb.repRate = 1; gb.polar = 1
    gb.sigX = sig; gb.sigY = sig; gb.sigT = 10e-15; gb.mx = 0; gb.my = 0
    w = L.SRWLWfr(); w.allocate(1, nx, ny)
    m = w.mesh
    m.zStart = z; m.eStart = E; m.eFin = E
    m.xStart, m.xFin, m.yStart, m.yFin = -xr, xr, -yr, yr
    w.partBeam.partStatMom1.x = 0.; w.partBeam.partStatMom1.y = 0.; w.partBeam.partStatMom1.z = 0.
    w.partBeam.partStatMom1.xp = 0.; w.partBeam.partStatMom1.yp = 0.
    L.srwl.CalcElecFieldGaussian(w, gb, [0])
    return w


def undulator_wfr(L, nx, ny, xr=1.5e-3, yr=1.5e-3, z=20., npTraj=20000):
    """Planar undulator (3 GeV, 0.5 A filament, 20 mm x 100 periods, K=1.5) first harmonic at z."""
    per, nper, K = 0.02, 100, 1.5
    By = K / (0.0934 * per * 1000.)
    und = L.SRWLMagFldU([L.SRWLMagFldH(1, 'v', By, 0, 1, 1)], per, nper)
    mag = L.SRWLMagFldC([und], array('d', [0]), array('d', [0]), array('d', [0]))
    eb = L.SRWLPartBeam()
    eb.Iavg = 0.5
    eb.partStatMom1.x = 0.; eb.partStatMom1.y = 0.
    eb.partStatMom1.z = -0.5 * per * (nper + 4)
    eb.partStatMom1.xp = 0.; eb.partStatMom1.yp = 0.
    eb.partStatMom1.gamma = 3. / 0.51099890221e-03
    gam2 = eb.partStatMom1.gamma ** 2
    lam1 = per / (2. * gam2) * (1. + K * K / 2.)
    E1 = 1.239842e-06 / lam1
    w = L.SRWLWfr(); w.allocate(1, nx, ny)
    m = w.mesh
    m.zStart = z; m.eStart = E1; m.eFin = E1
    m.xStart, m.xFin, m.yStart, m.yFin = -xr, xr, -yr, yr
    w.partBeam = eb
    L.srwl.CalcElecFieldSR(w, 0, mag, [1, 0.01, 0., 0., npTraj, 1, 0])
    return w


def impose_radius(w, R, dR):
    """Multiplies the field by exp(+i pi r^2/(lambda R)) and sets Rx=Ry=R, dRx=dRy=dR."""
    nx, ny = w.mesh.nx, w.mesh.ny
    x = np.linspace(w.mesh.xStart, w.mesh.xFin, nx)[None, :]
    y = np.linspace(w.mesh.yStart, w.mesh.yFin, ny)[:, None]
    lam = 1.239842e-06 / w.mesh.eStart
    ph = np.exp(1j * np.pi * (x * x + y * y) / (lam * R))
    for name in ('arEx', 'arEy'):
        a = np.array(getattr(w, name), np.float32)
        c = (a[0::2] + 1j * a[1::2]).reshape(ny, nx) * ph
        b = np.empty(2 * nx * ny, np.float32)
        b[0::2] = c.real.ravel(); b[1::2] = c.imag.ravel()
        setattr(w, name, array('f', b.tobytes()))
    w.Rx = w.Ry = R
    w.dRx = w.dRy = dR


def build_beamline(L, elems):
    opts = []
    for e in elems:
        if e[0] == 'drift':
            opts.append(L.SRWLOptD(e[1], e[2]) if len(e) > 2 else L.SRWLOptD(e[1]))
        elif e[0] == 'aperture':
            opts.append(L.SRWLOptA(e[1], e[2], e[3], e[4], e[5], e[6]))
        elif e[0] == 'lens':
            opts.append(L.SRWLOptL(e[1], e[2], e[3], e[4]))
        elif e[0] == 'transmission':
            tr, nx, ny, rx, ry, x, y, ext, Fx, Fy = e[1:11]
            ne, e0, e1 = (e[11:14] if len(e) > 11 else (1, 0., 0.))
            opts.append(L.SRWLOptT(nx, ny, rx, ry, array('d', np.asarray(tr, np.float64).tobytes()), ext, Fx, Fy, x, y,
                                   ne, e0, e1))
        elif e[0] == 'container':
            opts.append(L.SRWLOptC(build_beamline(L, e[1]), [list(map(float, p)) for p in e[2]]))
    return opts


def tr_table_e(nx, ny, rx, ry, x, y, F, ne, e0, e1):
    """A table vs photon energy, [ny][nx][ne] pairs: tr_table at each energy, scaled."""
    out = np.empty((ny, nx, ne, 2))
    for k in range(ne):
        t = tr_table(nx, ny, rx, ry, x, y, F * (1. + 0.1 * k), ripple=2e-11 * (1. + 0.5 * k), seed=10 + k)
        out[:, :, k, :] = t.reshape(ny, nx, 2)
    return out.ravel()


def tr_table(nx, ny, rx, ry, x, y, F, amp=0.3, ripple=3e-10, seed=0):
    """(T, OPD) pairs over [ny][nx]: a focusing optical path -(r^2)/(2F) with a seeded ripple and an
    amplitude transmission falling off towards the edges."""
    g = np.random.default_rng(seed)
    xs = x - 0.5 * rx + np.arange(nx) * (rx / (nx - 1))
    ys = y - 0.5 * ry + np.arange(ny) * (ry / (ny - 1))
    X, Y = np.meshgrid(xs - x, ys - y)
    kx, ky, ph = (2. * np.pi / rx) * g.uniform(1., 4.), (2. * np.pi / ry) * g.uniform(1., 4.), g.uniform(0., 6.)
    opd = -(X * X + Y * Y) / (2. * F) + ripple * np.sin(kx * X + ph) * np.cos(ky * Y)
    t = 1. - amp * (X * X / (0.25 * rx * rx) + Y * Y / (0.25 * ry * ry)) + 0.02 * g.standard_normal(X.shape)
    out = np.empty((ny, nx, 2))
    out[..., 0], out[..., 1] = t, opd
    return out.ravel()


def snapshot(w):
    ex = np.array(w.arEx, np.float32)
    ey = np.array(w.arEy, np.float32)
    m = w.mesh
    return dict(ex=ex, ey=ey,
                mesh=np.array([m.nx, m.ny, m.xStart, m.xFin, m.yStart, m.yFin, m.eStart, m.zStart], np.float64),
                scal=np.array([w.Rx, w.Ry, w.dRx, w.dRy, w.xc, w.yc, w.avgPhotEn, w.presCA], np.float64),
                momx=np.array(w.arMomX, np.float64)[:11], momy=np.array(w.arMomY, np.float64)[:11],
                prop=np.array(w.arElecPropMatr, np.float64)[:20])


PP0 = [0, 0, 1, 0, 0, 1., 1., 1., 1., 0, 0, 0]


def cases(L):
    """(name, wavefront factory, elements, propagation parameter lists)."""
    pp = lambda anal=0, pxm=1., pxd=1., pzm=1., pzd=1.: [0, 0, 1., anal, 0, pxm, pxd, pzm, pzd, 0, 0, 0]
    c0 = [('drift', 10., 0), ('aperture', 'r', 'a', 1e-3, 1e-3, 0., 0.), ('lens', 5., 5., 0., 0.), ('drift', 5., 0)]
    c1 = [('aperture', 'c', 'a', 0.8e-3, 0.8e-3, 0., 0.), ('lens', 10., 10., 0., 0.), ('drift', 10., 0)]
    c1pp = [pp(), pp(0, 2., 2., 2., 2.), pp(4)]
    c2 = [('drift', 30., 0), ('lens', 15., 15., 0., 0.), ('drift', 30., 0)]
    c2pp = [pp(2), pp(), pp(2)]
    # resize with its centre moved (pp[9] shift type: 1 x, 2 z, 3 both; pp[10], pp[11] the centre)
    ppo = lambda pxm, pxd, pzm, pzd, sh, xc, zc, anal=0: [0, 0, 1., anal, 0, pxm, pxd, pzm, pzd, sh, xc, zc]  # noqa: E731

    def g0(n):
        return lambda: gaussian_wfr(L, 1000., 50e-6, n, n, 1e-3, 1e-3)

    def g2(n, r):
        def f():
            w = gaussian_wfr(L, 10000., 20e-6, n, n, r, r)
            impose_radius(w, 30., 0.3)
            return w
        return f
    out = [
        ('c0_64', g0(64), c0, [PP0] * 4),
        ('c0_128', g0(128), c0, [PP0] * 4),
        ('c0_ragged_96x80', lambda: gaussian_wfr(L, 1000., 50e-6, 96, 80, 1e-3, 0.9e-3), c0, [PP0] * 4),
        ('c1_64', lambda: undulator_wfr(L, 64, 64, npTraj=4000), c1, c1pp),
        ('c1_96', lambda: undulator_wfr(L, 96, 96, npTraj=4000), c1, c1pp),
        ('c2_128', g2(128, 0.5e-3), c2, c2pp),
        # resize variants and edge cases of the mesh logic
        ('rs_shrink', g0(128), [('drift', 3., 0)], [pp(0, 0.5, 1., 0.5, 1.)]),
        ('rs_res_only', g0(64), [('drift', 3., 0)], [pp(0, 1., 2., 1., 1.5)]),
        ('rs_range_only', g0(64), [('drift', 3., 0)], [pp(0, 2., 1., 1.5, 1.)]),
        ('rs_post', g0(64), [('drift', 3., 0)], [pp(), pp(0, 1.3, 1.7, 1.2, 1.1)]),
        # off-centre resizing (sroptelm.cpp:2383-2433, TuneStepToKeepInterpLimitsTheSameAtResize
        # sroptel3.cpp:537): both axes growing; x shrinking in range while z stays; a range-only z
        # resize; centres near the edges (the new mesh reaches past both limits); a curved beam
        # (quadratic-term treatment) after a lens
        ('rs_offc_grow', g0(96), [('drift', 3., 0)], [ppo(1.5, 1.2, 1.3, 1.1, 3, 0.25e-3, -0.15e-3)]),
        ('rs_offc_shrink_x', g0(128), [('drift', 3., 0)], [ppo(0.7, 1.5, 1., 1., 1, -0.3e-3, 0.)]),
        ('rs_offc_range_z', g0(64), [('drift', 2., 0)], [ppo(1., 1., 1.6, 1., 2, 0., 0.4e-3)]),
        ('rs_offc_edge', g0(80), [('drift', 2., 0)], [ppo(1., 2., 1., 2., 3, 0.8e-3, -0.85e-3)]),
        ('rs_offc_quad', g2(96, 0.5e-3), [('lens', 15., 15., 0., 0.), ('drift', 10., 0)],
         [pp(), ppo(1.4, 1.3, 1.4, 1.3, 3, 0.05e-3, 0.02e-3)]),
        ('ob_circ_lens_offc', g0(96), [('aperture', 'c', 'o', 0.3e-3, 0.3e-3, 0.1e-3, 0.), ('drift', 2., 0),
                                      ('lens', 3., 4., 0.2e-3, -0.1e-3), ('drift', 2., 0)], [PP0] * 4),
        ('rect_ob_towaist', g2(96, 0.5e-3), [('aperture', 'r', 'o', 0.2e-3, 0.1e-3, 0., 0.), ('lens', 20., 20., 0., 0.),
                                             ('drift', 12., 0)], [pp(), pp(), pp(4)]),
        ('quad_neg_k', g2(96, 0.5e-3), [('drift', -45., 0)], [pp(2)]),
        ('treat_path', g0(64), [('drift', 2., 1)], [pp()]),
        # pp[3]=1: radius estimate from the rms divergence, on analytic moments, on moments an
        # aperture recomputed, and on a wavefront without moments (recomputed by the drift itself)
        ('quad1_c2', g2(128, 0.5e-3), c2, [pp(1), pp(), pp(1)]),
        ('quad1_clip', g2(96, 0.5e-3), [('aperture', 'r', 'a', 0.05e-3, 0.05e-3, 0., 0.), ('lens', 15., 15., 0., 0.),
                                        ('drift', 10., 0)], [pp(), pp(), pp(1)]),
        ('quad1_nomom', no_moments(lambda: undulator_wfr(L, 64, 64, npTraj=4000)), [('drift', 5., 0)], [pp(1)]),
        # pp[3]=3: from a waist over a large distance
        ('fromwaist_64', g0(64), [('drift', 20., 0)], [pp(3)]),
        ('fromwaist_lens_96x80', lambda: gaussian_wfr(L, 2000., 30e-6, 96, 80, 0.6e-3, 0.5e-3),
         [('drift', 6., 0), ('lens', 3., 3., 0., 0.), ('drift', 3., 0)], [pp(3), pp(), pp(3)]),
        # pp[3]=5: to a waist beyond the paraxial approximation (quadratic term kept, and taken off
        # first once an aperture's moment recomputation has set the treatment flags; path length)
        ('bpx_towaist', g2(96, 0.5e-3), [('lens', 15., 15., 0., 0.), ('drift', 30., 0)], [pp(), pp(5)]),
        ('bpx_clip', g2(96, 0.5e-3), [('aperture', 'r', 'a', 0.05e-3, 0.05e-3, 0., 0.), ('lens', 15., 15., 0., 0.),
                                      ('drift', 30., 0)], [pp(), pp(), pp(5)]),
        ('bpx_treat_offc', g2(96, 0.5e-3), [('lens', 15., 15., 0.02e-3, -0.01e-3), ('drift', 30., 1)],
         [pp(), pp(5)]),
        # generic transmission (SRWLOptT): a table narrower than the wavefront (zero outside), off
        # centre and on its own grid; the boundary values outside (extTr = 1) before a drift to the
        # waist; a table on exactly the wavefront's mesh (node snapping), then a lens and a drift
        ('tr_plate_offc', g2(96, 0.5e-3), [('transmission', tr_table(61, 53, 0.12e-3, 0.1e-3, 0.01e-3, -0.005e-3, 200.,
                                                                     ripple=2e-11),
                                            61, 53, 0.12e-3, 0.1e-3, 0.01e-3, -0.005e-3, 0, 200., 200.),
                                           ('drift', 10., 0)], [pp(), pp()]),
        ('tr_ext_towaist', g2(96, 0.5e-3), [('transmission', tr_table(40, 40, 0.1e-3, 0.1e-3, 0., 0., 200., ripple=2e-11,
                                                                      seed=1),
                                             40, 40, 0.1e-3, 0.1e-3, 0., 0., 1, 200., 200.), ('drift', 12., 0)],
         [pp(), pp(4)]),
        # nested containers: the outer entry's pre-resize before the container, its treatment for every
        # element inside (the inner lists, here with resizes and other drift modes, are not used);
        # a container inside a container
        ('nested_c0', g0(64), [('drift', 10., 0),
                               ('container', [('aperture', 'r', 'a', 1e-3, 1e-3, 0., 0.), ('lens', 5., 5., 0., 0.)],
                                [pp(0, 2., 2., 2., 2.), pp(3)]),
                               ('drift', 5., 0)], [pp(), pp(0, 1.25, 1.5, 1.25, 1.5), pp()]),
        ('nested_deep_quad', g2(96, 0.5e-3), [('container', [('drift', 10., 0),
                                                              ('container', [('lens', 15., 15., 0., 0.),
                                                                             ('drift', 20., 0)], [pp(0), pp(0)])],
                                               [pp(0), pp(0)])], [pp(2)]),
        # a table vs photon energy (ne = 3, the wavefront's energy between the 2nd and 3rd)
        ('tr_vs_energy', g2(96, 0.5e-3), [('transmission', tr_table_e(31, 27, 0.12e-3, 0.1e-3, 0., 0., 200., 3, 9000.,
                                                                      10400.),
                                           31, 27, 0.12e-3, 0.1e-3, 0., 0., 0, 200., 200., 3, 9000., 10400.),
                                          ('drift', 10., 0)], [pp(), pp()]),
        ('tr_aligned_lens', g0(64), [('transmission', tr_table(64, 64, 2e-3, 2e-3, 0., 0., 1e23, amp=0.1,
                                                               ripple=2e-10, seed=2),
                                      64, 64, 2e-3, 2e-3, 0., 0., 0, 1e23, 1e23), ('lens', 5., 5., 0., 0.),
                                     ('drift', 5., 0)], [pp(), pp(), pp()]),
    ]
    return out


def no_moments(make):
    """The wavefront of `make` with its statistical moments set to zero."""
    def f():
        w = make()
        w.arMomX = array('d', [0.] * 11)
        w.arMomY = array('d', [0.] * 11)
        return w
    return f


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--ref', default=os.environ.get('SRW_REFERENCE', '/root/reference'))
    a = ap.parse_args()
    L = load_reference(a.ref)
    # 1) good numbers
    probe = os.path.join(REPO, 'oracle', '_ref', 'nextfft_probe')
    txt = subprocess.run([probe, '300000'], capture_output=True, text=True, check=True).stdout
    with open(os.path.join(HERE, 'good_numbers.txt'), 'w') as f:
        f.write(txt)
    # 2) propagation cases
    blob = {}
    index = []
    for name, make, elems, pps in cases(L):
        w = make()
        # a 4x4 propagation matrix and vector to carry through the drifts (arElecPropMatr)
        w.arElecPropMatr = array('d', [1., 0.5, 0., 0., 0., 1., 0., 0., 0., 0., 1., -0.25, 0., 0., 0., 1.,
                                       1e-4, 2e-6, -3e-4, 4e-6])
        inp = snapshot(w)
        opt = L.SRWLOptC(build_beamline(L, elems), [list(map(float, p)) for p in pps])
        L.srwl.PropagElecField(w, opt)
        out = snapshot(w)
        for k, v in inp.items():
            blob[name + '/in/' + k] = v
        for k, v in out.items():
            blob[name + '/out/' + k] = v
        els = []
        for k, e in enumerate(elems):
            e = list(e)
            if e[0] == 'transmission':       # the table beside the case, named in the element
                key = '%s/tr%d' % (name, k)
                blob[key] = np.asarray(e[1], np.float64)
                e[1] = key
            els.append(e)
        index.append(dict(name=name, elements=els, props=[list(map(float, p)) for p in pps]))
        print(name, 'in', int(inp['mesh'][0]), int(inp['mesh'][1]), 'out', int(out['mesh'][0]), int(out['mesh'][1]),
              'R', out['scal'][0], out['scal'][1])
    # 3) intensity extraction (srwlCalcIntFromElecField vs x and y) on a propagated wavefront with both
    #    components: every polarisation, intensity / phase / Re / Im, and the averaging and adding modes
    wsrc = None
    for name, make, elems, pps in cases(L):
        if name == 'quad1_nomom':
            wsrc = make()
            L.srwl.PropagElecField(wsrc, L.SRWLOptC(build_beamline(L, elems), [list(map(float, p)) for p in pps]))
    nx, ny = wsrc.mesh.nx, wsrc.mesh.ny
    ex = np.array(wsrc.arEx, np.float32)
    xx = np.linspace(-1., 1., nx)[None, :]
    yy = np.linspace(-1., 1., ny)[:, None]
    c = (ex[0::2] + 1j * ex[1::2]).reshape(ny, nx) * (0.4 * np.exp(1j * (1.3 * xx - 0.7 * yy)) + 0.2 * xx)
    ey = np.empty(2 * nx * ny, np.float32)
    ey[0::2] = c.real.ravel(); ey[1::2] = c.imag.ravel()
    wsrc.arEy = array('f', ey.tobytes())
    blob['int/ex'] = ex
    blob['int/ey'] = ey
    blob['int/mesh'] = snapshot(wsrc)['mesh']
    ints = []
    for it in (0, 4, 5, 6):
        for pol in (0, 1, 2, 3, 4, 5, 6, -1, -2, -3, -4, -5):
            if pol < 0 and it != 0:
                continue
            n = nx * ny * (4 if pol == -5 else 1)
            for meth in (None, [1., 3.], [2.]):
                code = 'd' if it == 4 else 'f'
                prev = np.sin(np.arange(n) * 0.37).astype(np.float64 if it == 4 else np.float32)
                arI = array(code, prev.tobytes())
                args = [arI, wsrc, pol, it, 3, wsrc.mesh.eStart, 0., 0.]
                if meth is not None:
                    args.append(array('d', meth + [0.] * (20 - len(meth))))
                L.srwl.CalcIntFromElecField(*args)
                key = 'int/%d/%d/%d' % (it, pol, 0 if meth is None else int(meth[0]))
                blob[key] = np.array(arI, np.float64 if it == 4 else np.float32)
                ints.append(dict(key=key, int_type=it, pol=pol, meth=meth))
    blob['int/index'] = np.array(json.dumps(ints))
    # 3b) cuts vs x at y (dep 1), vs y at x (dep 2) and single points (dep 0): positions between nodes,
    #     on a node, within a step below the mesh start (extrapolation) and beyond the mesh end
    m = wsrc.mesh
    xs, ys = (m.xFin - m.xStart) / (nx - 1), (m.yFin - m.yStart) / (ny - 1)
    pos = [(m.xStart + 17.3 * xs, m.yStart + 40.6 * ys), (m.xStart + 31 * xs, m.yStart + 12 * ys),
           (m.xStart - 0.4 * xs, m.yStart - 0.7 * ys), (m.xFin + 2.5 * xs, m.yFin + 0.5 * ys)]
    cuts = []
    for it in (0, 4, 5, 6):
        for pol in (0, 1, 2, 3, 4, 5, 6, -1, -2, -3, -4, -5):
            if pol < 0 and it != 0:
                continue
            for dep in (0, 1, 2):
                for k, (x, y) in enumerate(pos):
                    n = {0: 1, 1: nx, 2: ny}[dep] * (4 if pol == -5 else 1)
                    code = 'd' if it == 4 else 'f'
                    arI = array(code, [0.] * n)
                    L.srwl.CalcIntFromElecField(arI, wsrc, pol, it, dep, wsrc.mesh.eStart, x, y)
                    key = 'icut/%d/%d/%d/%d' % (it, pol, dep, k)
                    blob[key] = np.array(arI, np.float64 if it == 4 else np.float32)
                    cuts.append(dict(key=key, int_type=it, pol=pol, dep=dep, x=x, y=y))
    blob['icut/index'] = np.array(json.dumps(cuts))
    # 4) Gaussian beams (srwlCalcElecFieldGaussian, precPar = [0]): waist at the observation plane,
    #    offsets / angles / Hermite modes / every polarisation, field units, spectral detuning
    gcases = [
        ('g_waist', dict(x=0., y=0., z=0., xp=0., yp=0., avgPhotEn=1000., pulseEn=0.001, repRate=1., polar=1,
                         sigX=50e-6, sigY=50e-6, sigT=10e-15, mx=0, my=0), dict(n=(64, 64), r=(1e-3, 1e-3), e=1000.,
                                                                                 z=0., unit=1)),
        ('g_modes_circ', dict(x=20e-6, y=-10e-6, z=-5., xp=5e-6, yp=-3e-6, avgPhotEn=3003., pulseEn=0.002,
                              repRate=10., polar=5, sigX=30e-6, sigY=20e-6, sigT=20e-15, mx=2, my=1),
         dict(n=(80, 64), r=(0.6e-3, 0.5e-3), e=3000., z=10., unit=2)),
        ('g_45_mode', dict(x=0., y=5e-6, z=1., xp=0., yp=0., avgPhotEn=2000., pulseEn=0.001, repRate=1., polar=3,
                           sigX=40e-6, sigY=25e-6, sigT=5e-15, mx=1, my=0), dict(n=(48, 56), r=(0.4e-3, 0.4e-3),
                                                                                e=2000., z=3., unit=1)),
        ('g_vert', dict(x=0., y=0., z=0., xp=1e-6, yp=0., avgPhotEn=1500., pulseEn=0.001, repRate=1., polar=2,
                        sigX=30e-6, sigY=30e-6, sigT=10e-15, mx=0, my=2), dict(n=(40, 40), r=(0.5e-3, 0.5e-3), e=1500.,
                                                                               z=2., unit=1)),
        ('g_135', dict(x=0., y=0., z=0., xp=0., yp=0., avgPhotEn=1500., pulseEn=0.001, repRate=1., polar=4,
                       sigX=30e-6, sigY=30e-6, sigT=10e-15, mx=0, my=0), dict(n=(40, 40), r=(0.5e-3, 0.5e-3), e=1500.,
                                                                              z=2., unit=1)),
        ('g_circ_left', dict(x=0., y=0., z=0., xp=0., yp=0., avgPhotEn=1500., pulseEn=0.001, repRate=1., polar=6,
                             sigX=30e-6, sigY=30e-6, sigT=10e-15, mx=1, my=1), dict(n=(40, 40), r=(0.5e-3, 0.5e-3),
                                                                                    e=1500., z=2., unit=1)),
    ]
    gidx = []
    for gname, gp, mp in gcases:
        gb = L.SRWLGsnBm()
        for k, v in gp.items():
            setattr(gb, k, v)
        w = L.SRWLWfr()
        w.allocate(1, mp['n'][0], mp['n'][1])
        m = w.mesh
        m.zStart = mp['z']; m.eStart = m.eFin = mp['e']
        m.xStart, m.xFin, m.yStart, m.yFin = -mp['r'][0], mp['r'][0], -mp['r'][1], mp['r'][1]
        w.unitElFld = mp['unit']
        w.arElecPropMatr = array('d', [0.] * 16 + [1e-4, 2e-6, -3e-4, 4e-6])
        L.srwl.CalcElecFieldGaussian(w, gb, [0])
        out = snapshot(w)
        for k, v in out.items():
            blob['gauss/' + gname + '/' + k] = v
        gidx.append(dict(name=gname, beam=gp, mesh=dict(nx=mp['n'][0], ny=mp['n'][1], xStart=-mp['r'][0],
                                                         xFin=mp['r'][0], yStart=-mp['r'][1], yFin=mp['r'][1],
                                                         eStart=mp['e'], eFin=mp['e'], zStart=mp['z']),
                         unit=mp['unit']))
    blob['gauss/index'] = np.array(json.dumps(gidx))
    # 5) intensities extracted during propagation (srwlPropagElecField's intList, flat format):
    #    after a drift, an aperture (mask still pending in the GPU plan), a lens, the last drift and
    #    the post-resize; intensity, Re E and Im E of several polarisations.  (The phase, type 4, is
    #    left out: the reference allocates the client array for it as float (AllocExtIntArray gets the
    #    converted type, sroptcnt.cpp:465, srradstr.cpp:807) and writes doubles into it, which crashes)
    pp = lambda anal=0, pxm=1., pxd=1., pzm=1., pzd=1.: [0, 0, 1., anal, 0, pxm, pxd, pzm, pzd, 0, 0, 0]  # noqa: E731
    c0 = [('drift', 10., 0), ('aperture', 'r', 'a', 1e-3, 1e-3, 0., 0.), ('lens', 5., 5., 0., 0.), ('drift', 5., 0)]
    c1 = [('aperture', 'c', 'a', 0.8e-3, 0.8e-3, 0., 0.), ('lens', 10., 10., 0., 0.), ('drift', 10., 0)]
    c1pp = [pp(), pp(0, 2., 2., 2., 2.), pp(4)]
    xcases = [
        ('x_c0', lambda: gaussian_wfr(L, 1000., 50e-6, 64, 64, 1e-3, 1e-3), c0, [PP0] * 4 + [pp(0, 1.5, 1., 1.25, 1.)],
         [(1, 6, 0), (2, 0, 5), (3, 6, 5), (3, 1, 6), (4, 2, 0), (5, 6, 0)]),
        ('x_c1', lambda: undulator_wfr(L, 64, 64, npTraj=4000), c1, c1pp,
         [(1, 6, 0), (2, -1, 0), (3, 6, 0), (3, 0, 6)]),
        # after a nested container (one element of the outer chain)
        ('x_nested', lambda: gaussian_wfr(L, 1000., 50e-6, 64, 64, 1e-3, 1e-3),
         [('drift', 10., 0), ('container', [('aperture', 'r', 'a', 1e-3, 1e-3, 0., 0.), ('lens', 5., 5., 0., 0.)],
                              [pp(), pp()]), ('drift', 5., 0)], [pp(), pp(0, 1.25, 1.5, 1.25, 1.5), pp()],
         [(2, 6, 0), (3, 1, 5)]),
    ]
    xidx = []
    for xname, make, elems, pps, reqs in xcases:
        w = make()
        if xname == 'x_c1':          # a vertical component too, so that the polarisations differ
            ex = np.array(w.arEx, np.float32)
            w.arEy = array('f', (0.3 * ex[::-1]).astype(np.float32).tobytes())
        inp = snapshot(w)
        intList = [[el, pol, typ, 3, 0, L.SRWLRadMesh(w.mesh.eStart, w.mesh.eStart, 1)] for el, pol, typ in reqs]
        L.srwl.PropagElecField(w, L.SRWLOptC(build_beamline(L, elems), [list(map(float, p)) for p in pps]), intList)
        for k, v in inp.items():
            blob['xint/' + xname + '/in/' + k] = v
        for i, it in enumerate(intList):
            m = it[5]
            blob['xint/%s/%d/mesh' % (xname, i)] = np.array([m.nx, m.ny, m.xStart, m.xFin, m.yStart, m.yFin, m.eStart,
                                                             m.ne], np.float64)
            blob['xint/%s/%d/I' % (xname, i)] = np.array(it[6], np.float64 if it[2] == 4 else np.float32)
        out = snapshot(w)
        blob['xint/' + xname + '/out/ex'] = out['ex']
        blob['xint/' + xname + '/out/mesh'] = out['mesh']
        xidx.append(dict(name=xname, elements=[list(e) for e in elems], props=[list(map(float, p)) for p in pps],
                         reqs=[list(r) for r in reqs]))
        print(xname, [int(blob['xint/%s/%d/mesh' % (xname, i)][0]) for i in range(len(reqs))])
    blob['xint/index'] = np.array(json.dumps(xidx))
    blob['index'] = np.array(json.dumps(index))
    np.savez_compressed(os.path.join(HERE, 'cases.npz'), **blob)


if __name__ == '__main__':
    main()
