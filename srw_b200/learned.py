"""Learned resize factors for the aperture -> lens -> drift beamlines.

The reference's users choose the range / resolution resize factors (pp[5..8] of the propagation
parameter lists: pxm, pxd, pzm, pzd; cpp/src/core/sroptcnt.cpp:307-316) by hand; too small factors
alias or under-resolve, too large ones waste memory and time (the propagated grid grows with the
product of range and resolution per axis).  This module learns them: a small MLP (64 x 64
downsampled intensity, fitted phase-curvature radii, the wavefront's extent and the element
parameters -> log2 of the four factors of the resize before the lens) is trained by the project's
own CUDA kernels (srwgMlp*: GEMM, bias + GELU, their gradients, MSE, Adam) on labels that sweeps of
the plain GPU propagation produce: for every training wavefront and axis, the cheapest factor pair
(by the autotuned per-length pass times, srw_b200.tune) whose intensity agrees with an oversampled
propagation within TOL_LABEL, the other axis held at the conservative factors; the combined label
is checked once more and replaced by the conservative factors when it fails.

At run time ``choose_factors`` rounds the prediction up to the factor grid and checks it: the
wavefront propagated with the chosen factors against the same wavefront with the conservative
factors (2, 2, 2, 2), relative L2 of the intensity on a common mesh; above the tolerance it falls
back to the conservative factors.  ``CheckedMultiE`` applies the same check to one electron of
every batch of a multi-electron run and runs the batch with the conservative factors when it fails.

    python -m srw_b200.learned --samples 20000 --out srw_b200/models/resize_mlp.npz   # GPU

torch provides device memory and streams only; every kernel is the library's.
"""
import argparse
import ctypes as C
import json
import math
import os
import threading
import time

import numpy as np

from . import capi

GRID_R = np.array([0.5, 0.625, 0.75, 1.0, 1.25, 1.5, 1.75, 2.0])   # candidate range factors
GRID_D = np.array([1.0, 1.25, 1.5, 1.75, 2.0])                     # candidate resolution factors
CONSERVATIVE = (2.0, 2.0, 2.0, 2.0)                                # pxm, pxd, pzm, pzd of the fallback
TOL_LABEL = 1e-3                                                   # relative L2 intensity error accepted
AXIS_TOL = 0.7 * TOL_LABEL                                         # per-axis share of it in the sweeps
N_IMG = 64 * 64
N_EXTRA = 13
N_IN = N_IMG + N_EXTRA
N_OUT = 4
HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_MODEL = os.path.join(HERE, 'models', 'resize_mlp.npz')


def ref_factors(n):
    """Factors of the oversampled propagation that labels are judged against (the grid stays within
    the 8192-point general-length limit)."""
    return (3.0, 3.0) if n <= 512 else (2.5, 2.5)


def _check(r, what):
    capi.check(r, what)


# ------------------------------------------------------------------------------------------------
# the network
# ------------------------------------------------------------------------------------------------
class ResizeMLP(object):
    """FP32 MLP n_in -> hidden... -> n_out, GELU between layers; weights W[l] (in x out), b[l]."""

    def __init__(self, n_in=N_IN, hidden=(256, 256, 256), n_out=N_OUT, device=0, seed=0):
        import torch
        self.torch = torch
        self.dev = torch.device('cuda', device)
        self.sizes = [n_in] + list(hidden) + [n_out]
        rng = np.random.default_rng(seed)
        self.W, self.b = [], []
        for a, c in zip(self.sizes[:-1], self.sizes[1:]):
            w = rng.standard_normal((a, c)).astype(np.float32) * np.float32(math.sqrt(2.0 / a))
            self.W.append(torch.from_numpy(w).to(self.dev))
            self.b.append(torch.zeros(c, dtype=torch.float32, device=self.dev))
        self.mW = [torch.zeros_like(w) for w in self.W]
        self.vW = [torch.zeros_like(w) for w in self.W]
        self.mb = [torch.zeros_like(b) for b in self.b]
        self.vb = [torch.zeros_like(b) for b in self.b]
        self.t = 0
        self.xmean = torch.zeros(n_in, device=self.dev)
        self.xscale = torch.ones(n_in, device=self.dev)

    def _st(self):
        return C.c_void_p(self.torch.cuda.current_stream(self.dev).cuda_stream)

    def forward(self, X):
        """X: [B, n_in] float32 CUDA tensor (already normalised).  Keeps what backward needs."""
        L = capi.lib()
        st = self._st()
        self.Z, self.Y = [], [X]
        a = X
        for l, (W, b) in enumerate(zip(self.W, self.b)):
            B, n_out = a.shape[0], W.shape[1]
            z = self.torch.empty((B, n_out), dtype=self.torch.float32, device=self.dev)
            _check(L.srwgMlpGemm(B, n_out, a.shape[1], a.data_ptr(), a.shape[1], 0, W.data_ptr(), n_out, 0,
                                 z.data_ptr(), n_out, 1.0, 0.0, st), 'mlp gemm')
            y = self.torch.empty_like(z)
            act = 1 if l + 1 < len(self.W) else 0
            _check(L.srwgMlpBiasAct(z.data_ptr(), b.data_ptr(), y.data_ptr(), B, n_out, act, st), 'mlp bias')
            self.Z.append(z)
            self.Y.append(y)
            a = y
        return a

    def backward(self, dOut):
        """Gradients of the last forward's inputs given dLoss/dOut; returns (dW list, db list)."""
        L = capi.lib()
        st = self._st()
        dW = [None] * len(self.W)
        db = [None] * len(self.W)
        d = dOut.contiguous()
        for l in range(len(self.W) - 1, -1, -1):
            act = 1 if l + 1 < len(self.W) else 0
            if act:
                _check(L.srwgMlpActBackward(self.Z[l].data_ptr(), d.data_ptr(), d.numel(), act, st), 'mlp act')
            a = self.Y[l]
            B, n_in, n_out = a.shape[0], a.shape[1], d.shape[1]
            gw = self.torch.empty((n_in, n_out), dtype=self.torch.float32, device=self.dev)
            _check(L.srwgMlpGemm(n_in, n_out, B, a.data_ptr(), n_in, 1, d.data_ptr(), n_out, 0, gw.data_ptr(),
                                 n_out, 1.0, 0.0, st), 'mlp dW')
            gb = self.torch.empty(n_out, dtype=self.torch.float32, device=self.dev)
            _check(L.srwgMlpColSum(d.data_ptr(), gb.data_ptr(), B, n_out, st), 'mlp db')
            dW[l], db[l] = gw, gb
            if l > 0:
                da = self.torch.empty((B, n_in), dtype=self.torch.float32, device=self.dev)
                W = self.W[l]
                _check(L.srwgMlpGemm(B, n_in, n_out, d.data_ptr(), n_out, 0, W.data_ptr(), n_out, 1, da.data_ptr(),
                                     n_in, 1.0, 0.0, st), 'mlp dA')
                d = da
        return dW, db

    def loss_grad(self, out, target):
        """Mean squared error and its gradient (srwgMlpMse)."""
        L = capi.lib()
        st = self._st()
        dout = self.torch.empty_like(out)
        loss = self.torch.zeros(1, dtype=self.torch.float64, device=self.dev)
        _check(L.srwgMlpMse(out.data_ptr(), target.data_ptr(), dout.data_ptr(), loss.data_ptr(), out.numel(), st),
               'mlp mse')
        return loss, dout

    def adam(self, dW, db, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        L = capi.lib()
        st = self._st()
        self.t += 1
        for p, g, m, v in zip(self.W + self.b, dW + db, self.mW + self.mb, self.vW + self.vb):
            _check(L.srwgMlpAdam(p.data_ptr(), g.data_ptr(), m.data_ptr(), v.data_ptr(), p.numel(), lr, b1, b2, eps,
                                 self.t, st), 'mlp adam')

    def set_normalisation(self, X):
        self.xmean = X.mean(0)
        self.xscale = X.std(0) + 1e-6

    def norm(self, X):
        return ((X - self.xmean) / self.xscale).contiguous()

    def predict(self, X):
        return self.forward(self.norm(X))

    def train(self, X, T, Xv=None, Tv=None, epochs=300, batch=128, lr=1e-3, seed=0, log=None):
        """Minibatch Adam on the MSE; returns the history [(epoch, train loss, validation loss)]."""
        torch = self.torch
        self.set_normalisation(X)
        Xn = self.norm(X)
        Xvn = self.norm(Xv) if Xv is not None else None
        g = torch.Generator(device='cpu').manual_seed(seed)
        hist = []
        n = X.shape[0]
        for ep in range(epochs):
            perm = torch.randperm(n, generator=g).to(self.dev)
            tot = 0.
            for i0 in range(0, n, batch):
                idx = perm[i0:i0 + batch]
                out = self.forward(Xn[idx].contiguous())
                loss, dout = self.loss_grad(out, T[idx].contiguous())
                dW, db = self.backward(dout)
                self.adam(dW, db, lr=lr)
                tot += float(loss.item()) * len(idx)
            vl = None
            if Xvn is not None:
                vl = float(self.loss_grad(self.forward(Xvn), Tv)[0].item())
            hist.append((ep, tot / n, vl))
            if log and (ep % 20 == 0 or ep == epochs - 1):
                log('epoch %d train %.5f val %s' % (ep, tot / n, vl))
        return hist

    def save(self, path, meta=None):
        os.makedirs(os.path.dirname(path), exist_ok=True)
        d = {'sizes': np.array(self.sizes), 'xmean': self.xmean.cpu().numpy(), 'xscale': self.xscale.cpu().numpy(),
             'meta': json.dumps(meta or {})}
        for l, (W, b) in enumerate(zip(self.W, self.b)):
            d['W%d' % l] = W.cpu().numpy()
            d['b%d' % l] = b.cpu().numpy()
        np.savez_compressed(path, **d)

    @classmethod
    def load(cls, path, device=0):
        d = np.load(path)
        sizes = [int(v) for v in d['sizes']]
        m = cls(sizes[0], tuple(sizes[1:-1]), sizes[-1], device=device)
        torch = m.torch
        for l in range(len(sizes) - 1):
            m.W[l] = torch.from_numpy(d['W%d' % l]).to(m.dev)
            m.b[l] = torch.from_numpy(d['b%d' % l]).to(m.dev)
        m.xmean = torch.from_numpy(d['xmean']).to(m.dev)
        m.xscale = torch.from_numpy(d['xscale']).to(m.dev)
        m.meta = json.loads(str(d['meta']))
        return m




# ------------------------------------------------------------------------------------------------
# features
# ------------------------------------------------------------------------------------------------
def features(ex, ey, mesh, energy, ap, f, L, torch_dev, Rx=0., Ry=0.):
    """Feature vector of one wavefront (complex64 CUDA tensors [ny, nx]) and its beamline: the 64 x 64
    intensity (srwgWfrFeatures) normalised to its maximum and square-rooted, the fitted curvature
    radii (as 1/R [1/m]; the wavefront's own radii Rx, Ry are removed before the fit and added
    back), photon energy, the aperture (shape, Dx, Dy relative to the wavefront's extent), f, L, the
    extent and the number of points per axis."""
    import torch
    ny, nx = ex.shape
    xs = (mesh['xFin'] - mesh['xStart']) / (nx - 1)
    zs = (mesh['yFin'] - mesh['yStart']) / (ny - 1)
    feat = torch.empty(N_IMG, dtype=torch.float32, device=torch_dev)
    sums = torch.zeros(4, dtype=torch.float64, device=torch_dev)
    st = C.c_void_p(torch.cuda.current_stream(torch_dev).cuda_stream)
    k = 2. * math.pi / (1.239842e-06 / energy)
    i0x = 1. / Rx if Rx != 0. else 0.
    i0z = 1. / Ry if Ry != 0. else 0.
    _check(capi.lib().srwgWfrFeatures(ex.data_ptr(), ey.data_ptr(), nx, ny, mesh['xStart'], xs, mesh['yStart'], zs,
                                      k, i0x, i0z, feat.data_ptr(), sums.data_ptr(), st), 'features')
    s = sums.cpu().numpy()
    invRx = i0x + (s[0] / (k * xs * s[1]) if s[1] > 0 else 0.)     # dphi ~ k x dx / R
    invRz = i0z + (s[2] / (k * zs * s[3]) if s[3] > 0 else 0.)
    img = torch.sqrt(feat / torch.clamp(feat.max(), min=1e-30))
    wx = mesh['xFin'] - mesh['xStart']
    wz = mesh['yFin'] - mesh['yStart']
    shape, dx, dz = ap
    extra = torch.tensor([invRx, invRz, math.log(energy / 1000.), dx / wx, dz / wz, 1. if shape == 'r' else 0.,
                          math.log(f), math.log(L), math.log(L / f), math.log(wx * 1e3), math.log(wz * 1e3),
                          math.log2(nx), math.log2(ny)], dtype=torch.float32, device=torch_dev)
    return torch.cat([img, extra])


# ------------------------------------------------------------------------------------------------
# synthetic wavefronts and beamlines (Gaussian and undulator-like, 1-20 keV, drifts 1-50 m,
# f 1-30 m, circular and rectangular apertures 0.1-2 mm)
# ------------------------------------------------------------------------------------------------
def sample_case(rng, n=None):
    if n is None:
        u = rng.random()
        n = 256 if u < 0.45 else (512 if u < 0.9 else 1024)
    E = math.exp(rng.uniform(math.log(1000.), math.log(20000.)))
    lam = 1.239842e-06 / E
    z = math.exp(rng.uniform(math.log(5.), math.log(50.)))              # source -> first element
    if rng.random() < 0.5:
        sx0 = math.exp(rng.uniform(math.log(5e-6), math.log(60e-6)))       # waist rms, x
        sz0 = sx0 * math.exp(rng.uniform(-0.5, 0.5))                       # and z
        def prop(s0):
            zr = 4. * math.pi * s0 * s0 / lam
            return s0 * math.sqrt(1. + (z / zr) ** 2), z * (1. + (zr / z) ** 2)
        (sx, Rx), (sz, Rz) = prop(sx0), prop(sz0)
        rx, rz = 4. * sx, 4. * sz
        x, y = np.linspace(-rx, rx, n), np.linspace(-rz, rz, n)
        X, Y = np.meshgrid(x, y)
        ex = np.exp(-X * X / (4. * sx * sx) - Y * Y / (4. * sz * sz)) * \
            np.exp(1j * math.pi * (X * X / Rx + Y * Y / Rz) / lam)
        kind = 'gaussian'
    else:
        nper = int(rng.integers(40, 200))
        rx = z * math.sqrt(3. * lam / (nper * 0.02)) * rng.uniform(0.8, 1.6)   # ~ a few rings of the harmonic
        rz = rx * math.exp(rng.uniform(-0.3, 0.3))
        x, y = np.linspace(-rx, rx, n), np.linspace(-rz, rz, n)
        X, Y = np.meshgrid(x, y)
        th2 = (X * X + Y * Y) / (z * z)
        q = th2 * nper * 0.02 / (2. * lam)                              # detuning of the first harmonic
        ex = np.sinc(q) * np.exp(-1j * math.pi * q) * np.exp(1j * math.pi * (X * X + Y * Y) / (lam * z))
        Rx = Rz = z
        kind = 'undulator'
    ex = (ex * 1e6).astype(np.complex64)
    ey = np.zeros_like(ex)
    mesh = dict(nx=n, ny=n, xStart=-rx, xFin=rx, yStart=-rz, yFin=rz, eStart=E, eFin=E, zStart=z)
    sc = dict(Rx=Rx, Ry=Rz, dRx=0.01 * Rx, dRy=0.01 * Rz)
    if rng.random() < 0.5:
        d = min(2e-3, max(1e-4, 2. * min(rx, rz) * rng.uniform(0.3, 0.9)))
        ap = ('c', d, d)
    else:
        ap = ('r', min(2e-3, max(1e-4, 2. * rx * rng.uniform(0.3, 0.9))),
              min(2e-3, max(1e-4, 2. * rz * rng.uniform(0.3, 0.9))))
    f = math.exp(rng.uniform(math.log(1.), math.log(30.)))
    L = f * math.exp(rng.uniform(-0.3, 0.3))
    L = min(50., max(1., L))
    return dict(kind=kind, ex=ex, ey=ey, mesh=mesh, sc=sc, E=E, ap=ap, f=f, L=L, drift_mode=4)


def bench_case(ex, ey, mesh, sc, ap_d=0.8e-3, f=10., L=10.):
    """The undulator benchmark beamline's wavefront and elements as a case of this module."""
    return dict(kind='undulator', ex=ex, ey=ey, mesh=mesh, sc=sc, E=mesh['eStart'], ap=('c', ap_d, ap_d), f=f, L=L,
                drift_mode=4)


def beamline(mod, ap, f, L, fac, drift_mode=4):
    """aperture -> (resize fac = (pxm, pxd, pzm, pzd)) lens -> drift (to the waist by default)."""
    pp = lambda anal=0, fc=(1., 1., 1., 1.): [0, 0, 1., anal, 0, fc[0], fc[1], fc[2], fc[3], 0, 0, 0]  # noqa: E731
    return mod.SRWLOptC([mod.SRWLOptA(ap[0], 'a', ap[1], ap[2]), mod.SRWLOptL(f, f), mod.SRWLOptD(L)],
                        [pp(), pp(0, tuple(fac)), pp(drift_mode)])


def _wfr(mod, case):
    w = mod.SRWLWfr()
    n = case['mesh']['nx']
    w.allocate(1, n, case['mesh']['ny'])
    for name, fld in (('arEx', case['ex']), ('arEy', case['ey'])):
        a = np.empty(2 * fld.size, np.float32)
        a[0::2] = fld.real.ravel()
        a[1::2] = fld.imag.ravel()
        setattr(w, name, a)
    for k in ('xStart', 'xFin', 'yStart', 'yFin', 'eStart', 'eFin', 'zStart'):
        setattr(w.mesh, k, case['mesh'][k])
    w.Rx, w.Ry, w.dRx, w.dRy = case['sc']['Rx'], case['sc']['Ry'], case['sc']['dRx'], case['sc']['dRy']
    return w


def _interp_cubic(I, om, em, torch):
    """I at the points of mesh em by 4 x 4 cubic Lagrange interpolation (nodes -1..2 around the
    cell, as RadResizeCore's interpolation; the cell is clamped at the edges; zero outside)."""
    ny, nx = I.shape
    xs = (om['xFin'] - om['xStart']) / (nx - 1)
    ys = (om['yFin'] - om['yStart']) / (ny - 1)
    xa = em['xStart'] + torch.arange(em['nx'], dtype=torch.float64, device=I.device) * (em['xFin'] - em['xStart']) / (em['nx'] - 1)
    ya = em['yStart'] + torch.arange(em['ny'], dtype=torch.float64, device=I.device) * (em['yFin'] - em['yStart']) / (em['ny'] - 1)

    def axis(f, n):
        i = torch.floor(f).long()
        ok = (i >= 0) & (i < n - 1)
        st = (i - 1).clamp(0, n - 4)
        t = f - (st + 1)
        w = torch.stack([-t * (t - 1) * (t - 2) / 6, (t + 1) * (t - 1) * (t - 2) / 2, -(t + 1) * t * (t - 2) / 2,
                         (t + 1) * t * (t - 1) / 6], 1)
        return st, w, ok

    sx, wx, okx = axis((xa - om['xStart']) / xs, nx)
    sy, wy, oky = axis((ya - om['yStart']) / ys, ny)
    rows = torch.zeros((em['ny'], nx), dtype=I.dtype, device=I.device)
    for a in range(4):
        rows += wy[:, a:a + 1] * I[sy + a]
    out = torch.zeros((em['ny'], em['nx']), dtype=I.dtype, device=I.device)
    for a in range(4):
        out += wx[:, a].unsqueeze(0) * rows[:, sx + a]
    return out * (oky.unsqueeze(1) & okx.unsqueeze(0))


def propagate_intensity(case, fac, dev, stream=None):
    """Plain GPU propagation with factors fac = (pxm, pxd, pzm, pzd): (total intensity [ny, nx]
    float64 CUDA, mesh)."""
    import torch
    from . import srwlib as mod
    from .plan import Plan
    w = _wfr(mod, case)
    p = Plan(w, beamline(mod, case['ap'], case['f'], case['L'], fac, case.get('drift_mode', 4)), device=dev.index)
    ex = torch.from_numpy(case['ex']).to(dev)
    ey = torch.from_numpy(case['ey']).to(dev)
    ox, oy = p.new_output()
    p.execute(ex, ey, ox, oy, stream)
    I = (ox.real.double() ** 2 + ox.imag.double() ** 2 + oy.real.double() ** 2 + oy.imag.double() ** 2)
    return I, p.output_mesh()


def eval_box(I_ref, om):
    """Box around the reference intensity that holds its points above 1e-3 of the maximum."""
    import torch
    m = I_ref > 1e-3 * I_ref.max()
    ny, nx = I_ref.shape
    ys = torch.nonzero(m.any(1)).flatten()
    xs = torch.nonzero(m.any(0)).flatten()
    fx = lambda i: om['xStart'] + (om['xFin'] - om['xStart']) * float(i) / (nx - 1)   # noqa: E731
    fy = lambda i: om['yStart'] + (om['yFin'] - om['yStart']) * float(i) / (ny - 1)   # noqa: E731
    return fx(xs.min()), fx(xs.max()), fy(ys.min()), fy(ys.max())


def factor_error(I, om, I_ref, om_ref, box):
    """Relative L2 intensity error of a propagation at its own output nodes inside `box`, against
    the reference propagation interpolated to those nodes by cubic Lagrange interpolation; 1 when
    the output window does not cover the box."""
    import torch
    x0, x1, y0, y1 = box
    if om['xStart'] > x0 or om['xFin'] < x1 or om['yStart'] > y0 or om['yFin'] < y1:
        return 1.0
    ny, nx = I.shape
    xs = (om['xFin'] - om['xStart']) / (nx - 1)
    ys = (om['yFin'] - om['yStart']) / (ny - 1)
    i0, i1 = int(math.ceil((x0 - om['xStart']) / xs)), int(math.floor((x1 - om['xStart']) / xs))
    j0, j1 = int(math.ceil((y0 - om['yStart']) / ys)), int(math.floor((y1 - om['yStart']) / ys))
    if i1 <= i0 or j1 <= j0:
        return 1.0
    sub = dict(nx=i1 - i0 + 1, ny=j1 - j0 + 1, xStart=om['xStart'] + i0 * xs, xFin=om['xStart'] + i1 * xs,
               yStart=om['yStart'] + j0 * ys, yFin=om['yStart'] + j1 * ys)
    ref = _interp_cubic(I_ref, om_ref, sub, torch)
    c = I[j0:j1 + 1, i0:i1 + 1]
    return float(torch.linalg.norm(c - ref) / torch.linalg.norm(ref))


# ------------------------------------------------------------------------------------------------
# cost model: autotuned per-length pass times (srw_b200.tune), per point
# ------------------------------------------------------------------------------------------------
_TIMES = None


def _times():
    global _TIMES
    if _TIMES is None:
        from . import tune
        _TIMES = tune.load_times()
    return _TIMES


def new_length(n, rf, df):
    """Resized number of points: round-half-up of n rf df (RadResizeGen), then the next good FFT
    number (NextCorrectNumberForFFT, gmfft.cpp:156), n itself when both factors are within 1e-4 of 1."""
    if abs(rf - 1.) < 1e-4 and abs(df - 1.) < 1e-4:
        return n
    return int(capi.lib().srwgNextFftNumber(int(math.floor(n * rf * df + 0.5))))


FILLED = 1024            # shortest line length whose single-wavefront passes fill the GPU


def point_costs(n):
    """(row, column) pass time per point [ms] of length n from the tuning table.  The table times
    one wavefront; below FILLED points per line its passes are too small to fill the GPU and the
    time is mostly launch and tail latency, which a batch of wavefronts does not pay per wavefront,
    so there the per-point time of the shortest measured length from FILLED up of the same kind
    (power of two or not) stands in.  A length the table lacks gets the largest per-point time of
    its measured neighbours times 3 (the run-time-scheduled kernel)."""
    t = _times()
    if not t:
        return (1., 1.) if (n & (n - 1)) == 0 else (5., 5.)
    pow2 = (n & (n - 1)) == 0
    if n < FILLED:
        same = sorted(m for m in t if m >= FILLED and ((m & (m - 1)) == 0) == pow2)
        if same:
            m = same[0]
            return t[m][0] / (m * m), t[m][1] / (m * m)
    if n in t:
        return t[n][0] / (n * n), t[n][1] / (n * n)
    near = sorted(t, key=lambda m: abs(math.log(m / n)))[:3]
    return (3. * max(t[m][0] / (m * m) for m in near), 3. * max(t[m][1] / (m * m) for m in near))


def grid_cost(nx, nz, fac):
    """Modelled time of propagating an nx x nz wavefront with factors fac: the row and column
    passes on the resized grid (per-point times of its lengths) plus the resize (proportional to
    the points written, at the row-pass rate)."""
    mx, mz = new_length(nx, fac[0], fac[1]), new_length(nz, fac[2], fac[3])
    r, _ = point_costs(mx)
    _, c = point_costs(mz)
    return mx * mz * (r + c) + mx * mz * r


def _pairs():
    return [(float(r), float(d)) for r in GRID_R for d in GRID_D]


def choose_grid(pred, nx, nz):
    """Prediction (log2 of pxm, pxd, pzm, pzd) -> the cheapest grid factors (grid_cost) with every
    factor not below the prediction (per axis)."""
    lo = [2. ** float(v) - 1e-6 for v in pred]
    px = [p for p in _pairs() if p[0] >= lo[0] and p[1] >= lo[1]] or [CONSERVATIVE[:2]]
    pz = [p for p in _pairs() if p[0] >= lo[2] and p[1] >= lo[3]] or [CONSERVATIVE[2:]]
    best, bc = CONSERVATIVE, None
    for a in px:
        for b in pz:
            c = grid_cost(nx, nz, a + b)
            if bc is None or c < bc:
                best, bc = tuple(a) + tuple(b), c
    return best


# ------------------------------------------------------------------------------------------------
# labels
# ------------------------------------------------------------------------------------------------
def label_case(case, dev, stream=None):
    import torch
    """Cheapest factors (pxm, pxd, pzm, pzd) within tolerance of the oversampled propagation: per
    axis the candidate pairs in order of the resized length (the other axis at the conservative
    factors), the first within AXIS_TOL found by bisection; the combination is checked against
    TOL_LABEL and replaced by the conservative factors when it fails.  Returns (factors, error of
    the label, evaluations)."""
    n = case['mesh']['nx']
    rf = ref_factors(n)
    Iref, omref = propagate_intensity(case, rf + rf, dev, stream)
    mx = float(Iref.max())
    if not math.isfinite(mx) or mx <= 0. or not bool(torch.isfinite(Iref).all()):
        raise ValueError('no usable reference intensity (aperture blocks the beam?)')
    box = eval_box(Iref, omref)
    cache = {}

    def err(fac):
        if fac not in cache:
            I, om = propagate_intensity(case, fac, dev, stream)
            cache[fac] = factor_error(I, om, Iref, omref, box)
        return cache[fac]

    best = []
    for axis in (0, 1):
        nn = case['mesh']['nx'] if axis == 0 else case['mesh']['ny']
        full = new_length(nn, *CONSERVATIVE[:2])
        cands = [p for p in sorted(_pairs(), key=lambda p: (new_length(nn, *p), p[1], p[0]))
                 if new_length(nn, *p) < full]

        def ok(p):
            fac = (p + CONSERVATIVE[2:]) if axis == 0 else (CONSERVATIVE[:2] + p)
            return err(fac) <= AXIS_TOL
        # the error falls as the resized length grows: bisect for the first candidate within the
        # tolerance, then walk up from there while the neighbours disagree with that assumption
        lo, hi = 0, len(cands)
        while lo < hi:
            mid = (lo + hi) // 2
            if ok(cands[mid]):
                hi = mid
            else:
                lo = mid + 1
        while lo < len(cands) and not ok(cands[lo]):
            lo += 1
        best.append(tuple(cands[lo]) if lo < len(cands) else tuple(CONSERVATIVE[:2]))
    lab = best[0] + best[1]
    e = err(lab)
    if e > TOL_LABEL:
        lab, e = CONSERVATIVE, err(CONSERVATIVE)
    return lab, e, len(cache) + 1


def case_features(case, dev):
    import torch
    ex = torch.from_numpy(case['ex']).to(dev)
    ey = torch.from_numpy(case['ey']).to(dev)
    return features(ex, ey, case['mesh'], case['E'], case['ap'], case['f'], case['L'], dev, case['sc']['Rx'],
                    case['sc']['Ry'])


def target(factors):
    return np.log2(np.array(factors, np.float32))


# ------------------------------------------------------------------------------------------------
# run time
# ------------------------------------------------------------------------------------------------
def _common_error(I, om, I_c, om_c):
    """Relative L2 of intensity I (mesh om) against I_c (mesh om_c, the conservative propagation)
    at om's nodes inside the box where I_c exceeds 1e-3 of its maximum."""
    return factor_error(I, om, I_c, om_c, eval_box(I_c, om_c))


def on_mesh(I, om, em):
    """Intensity I (torch float64 [ny, nx] on mesh om) interpolated bilinearly at the nodes of mesh em,
    zero outside om, as the multi-electron accumulation does (avg_update_interp, order 1)."""
    import torch
    ny, nx = I.shape
    xs = (om['xFin'] - om['xStart']) / (nx - 1)
    ys = (om['yFin'] - om['yStart']) / (ny - 1)
    xa = em['xStart'] + torch.arange(em['nx'], dtype=torch.float64, device=I.device) * (em['xFin'] - em['xStart']) / (em['nx'] - 1)
    ya = em['yStart'] + torch.arange(em['ny'], dtype=torch.float64, device=I.device) * (em['yFin'] - em['yStart']) / (em['ny'] - 1)
    ix = torch.trunc((xa - om['xStart']) / xs + 1.e-09).long()
    iy = torch.trunc((ya - om['yStart']) / ys + 1.e-09).long()
    okx = (ix >= 0) & (ix < nx - 1)
    oky = (iy >= 0) & (iy < ny - 1)
    ix, iy = ix.clamp(0, nx - 2), iy.clamp(0, ny - 2)
    tx = ((xa - (om['xStart'] + xs * ix)) / xs).unsqueeze(0)
    ty = ((ya - (om['yStart'] + ys * iy)) / ys).unsqueeze(1)
    a00, f10 = I[iy][:, ix], I[iy][:, ix + 1]
    f01, f11 = I[iy + 1][:, ix], I[iy + 1][:, ix + 1]
    v = a00 + tx * ((f10 - a00) + ty * (a00 - f01 - f10 + f11)) + ty * (f01 - a00)
    return v * (oky.unsqueeze(1) & okx.unsqueeze(0))


def mesh_error(I, om, I_c, om_c, em):
    """Relative L2 of intensity I (mesh om) against the conservative one I_c (mesh om_c), both
    interpolated onto the detector mesh em, where I_c exceeds 1e-3 of its maximum there."""
    import torch
    a, b = on_mesh(I, om, em), on_mesh(I_c, om_c, em)
    sel = b > 1e-3 * b.max()
    return float(torch.linalg.norm((a - b)[sel]) / torch.linalg.norm(b[sel]))


def _next(grid, v):
    larger = grid[grid > v + 1e-9]
    return float(larger[0]) if len(larger) else float(v)


def mean_intensity(case, fac, offsets, acc_mesh, dev):
    """Mean intensity (torch float64 [ny, nx] on dev) on mesh acc_mesh of the electrons `offsets`
    ([n, 4] or [n, 5], srw_b200.multie.MultiE): the case's wavefront offset per electron,
    propagated with factors fac."""
    import torch
    from . import srwlib as mod
    from .multie import MultiE
    acc = torch.zeros((acc_mesh['ny'], acc_mesh['nx']), dtype=torch.float64, device=dev)
    me = MultiE(_wfr(mod, case), beamline(mod, case['ap'], case['f'], case['L'], fac, case.get('drift_mode', 4)),
                acc_mesh, max_batch=min(16, len(offsets)), graph=False, device=dev.index)
    me.use_accumulator(acc.data_ptr())
    me.add(offsets, torch.cuda.current_stream(dev).cuda_stream)
    torch.cuda.synchronize(dev)
    del me
    return acc / len(offsets)


def rel_err(a, ref):
    """Relative L2 of intensity a against ref (same mesh) where ref exceeds 1e-3 of its maximum."""
    import torch
    sel = ref > 1e-3 * ref.max()
    d = torch.linalg.norm(ref[sel])
    return float(torch.linalg.norm((a - ref)[sel]) / d) if float(d) > 0. else float('inf')


def candidates_from(fac, tries, nx=None, nz=None):
    """Candidates for the check, in order: the prediction rounded to the grid, then the prediction
    with its range factors raised 1, 2, 3 grid steps and its resolution factors 0 or 1 step (range sets
    the output mesh step of a propagation to the waist, resolution its extent), cheapest first (grid
    cost on an nx x nz input when given), none as dear as the conservative factors; at most `tries`."""
    rx, dx, rz, dz = fac
    out = [tuple(fac)]
    more = []
    for sr in (1, 2, 3):
        for sd in (0, 1):
            ax, az, bx, bz = rx, rz, dx, dz
            for _ in range(sr):
                ax, az = _next(GRID_R, ax), _next(GRID_R, az)
            for _ in range(sd):
                bx, bz = _next(GRID_D, bx), _next(GRID_D, bz)
            more.append((ax, bx, az, bz))
    if nx is not None:
        cmax = grid_cost(nx, nz, CONSERVATIVE)
        more = sorted((c for c in more if grid_cost(nx, nz, c) < cmax), key=lambda c: grid_cost(nx, nz, c))
    for c in more:
        if c not in out and c != tuple(CONSERVATIVE):
            out.append(c)
    return out[:tries]


def _prev(grid, v):
    smaller = grid[grid < v - 1e-9]
    return float(smaller[-1]) if len(smaller) else float(v)


def choose_factors(model, case, dev, check_tol=TOL_LABEL, acc_mesh=None, tries=6, check_offsets=None, trace=None,
                   refine=0):
    """(factors, used_fallback, check_error): the network's factors, rounded up to the grid, checked
    against the conservative factors; when the check exceeds check_tol, the candidates of
    candidates_from (range raised first, cheapest first; up to `tries` in all) follow before the
    conservative factors are used.  With refine > 0, a passing choice is then refined by the check:
    its resolution factors lowered a grid step at a time (both axes, then x alone, then z alone) while
    the check still passes, at most `refine` more checks.

    The check compares what the run produces.  With check_offsets (electrons [n, 4|5], and acc_mesh)
    it is the mean intensity of those electrons on the detector mesh acc_mesh, propagated with the
    candidate and with the conservative factors (a multi-electron run's result); otherwise the
    wavefront itself, relative L2 of the intensity on acc_mesh when given, else at the candidate's
    output nodes.  `trace`, a list, receives (factors, error) of every candidate checked."""
    feat = case_features(case, dev).unsqueeze(0)
    pred = model.predict(feat)[0].cpu().numpy()
    fac = tuple(choose_grid(pred, case['mesh']['nx'], case['mesh']['ny']))
    if fac == tuple(CONSERVATIVE):
        return CONSERVATIVE, False, 0.
    if check_offsets is not None:
        if acc_mesh is None:
            raise ValueError('a check on electrons needs the detector mesh')
        Ic = mean_intensity(case, CONSERVATIVE, check_offsets, acc_mesh, dev)
    else:
        Ic, omc = propagate_intensity(case, CONSERVATIVE, dev)

    def check(c):
        if check_offsets is not None:
            e = rel_err(mean_intensity(case, c, check_offsets, acc_mesh, dev), Ic)
        else:
            I, om = propagate_intensity(case, c, dev)
            e = mesh_error(I, om, Ic, omc, acc_mesh) if acc_mesh is not None else _common_error(I, om, Ic, omc)
        if trace is not None:
            trace.append((c, e))
        return e

    e, got = None, None
    for c in candidates_from(fac, tries, case['mesh']['nx'], case['mesh']['ny']):
        if c == tuple(CONSERVATIVE):
            break
        e = check(c)
        if e <= check_tol:
            got = c
            break
    if got is None:
        return CONSERVATIVE, True, e
    left = refine
    while left > 0:
        rx, dx, rz, dz = got
        better = False
        for c in ((rx, _prev(GRID_D, dx), rz, _prev(GRID_D, dz)), (rx, _prev(GRID_D, dx), rz, dz),
                  (rx, dx, rz, _prev(GRID_D, dz))):
            if c == got or left <= 0:
                continue
            left -= 1
            e2 = check(c)
            if e2 <= check_tol:
                got, e, better = c, e2, True
                break
        if not better:
            break
    return got, False, e


class CheckedMultiE(object):
    """Multi-electron propagation (srw_b200.multie.MultiE) with learned factors and a run-time check
    of the mean intensity.  A check set of electrons is propagated with both the learned and the
    conservative factors into two FP64 sums on the detector mesh: the electrons `check_offsets`
    given at construction (those of choose_factors' check), then the first electron of every batch.
    With every batch the relative L2 of the two sums (where the conservative one exceeds 1e-3 of its
    maximum) is queued on the stream behind the batch; it is read before the batch after next is
    queued, or by ``mean()``, so the host never waits for the batch it has just queued.  Above `tol`
    the run falls back for good: every electron added so far with the learned factors (the checked
    batch and the one after it included) is propagated again with the conservative ones (the sum is
    rebuilt), and so are all later batches.
    ``mean()`` divides by the electrons added."""

    def __init__(self, base_wfr, make_beamline, factors, acc_mesh, max_batch=64, safe_batch=16, graph=True,
                 device=0, tol=TOL_LABEL, check_offsets=None, launch_batch=None):
        import torch
        from .multie import MultiE, offset_array
        self.torch = torch
        self.dev = torch.device('cuda', device)
        self.acc = torch.zeros((acc_mesh['ny'], acc_mesh['nx']), dtype=torch.float64, device=self.dev)
        self.chk = [torch.zeros_like(self.acc), torch.zeros_like(self.acc)]
        self.learned = tuple(factors) != tuple(CONSERVATIVE)
        # a checked batch of max_batch electrons runs as launches of launch_batch electrons (default: one
        # launch), so that the device starts on the first launch while the host plans the next
        self.fast = MultiE(base_wfr, make_beamline(factors), acc_mesh, max_batch=launch_batch or max_batch,
                           graph=graph, device=device)
        self.safe = MultiE(base_wfr, make_beamline(CONSERVATIVE), acc_mesh, max_batch=safe_batch, graph=graph,
                           device=device)
        self.fast.use_accumulator(self.acc.data_ptr())
        self.safe.use_accumulator(self.acc.data_ptr())
        self.cfast = self.csafe = None
        if self.learned:
            self.cfast = MultiE(base_wfr, make_beamline(factors), acc_mesh, max_batch=16, graph=False, device=device)
            self.csafe = MultiE(base_wfr, make_beamline(CONSERVATIVE), acc_mesh, max_batch=16, graph=False,
                                device=device)
            self.cfast.use_accumulator(self.chk[0].data_ptr())
            self.csafe.use_accumulator(self.chk[1].data_ptr())
        self.check0 = None if check_offsets is None else offset_array(check_offsets)
        self.max_batch, self.tol = max_batch, tol
        # pinned read-back slots of the queued checks (at most two are in flight: see add)
        self._hosts = [torch.empty(2, dtype=torch.float64, pin_memory=True) for _ in range(3)]
        self._next_host = 0
        # the batches, the checks and the fallback run on this stream when the caller gives none, so
        # that the host plans the next batch while the device runs the last one
        self._stream = torch.cuda.Stream(self.dev)
        self._start()

    def _start(self):
        self.n, self.n_check, self.batches, self.check_errors = 0, 0, 0, []
        self.fell_back, self.rerun, self.added_fast = False, 0, []
        self._pending = []                         # queued checks, oldest first: (event, host slot)
        for c in self.chk:
            c.zero_()
        self.torch.cuda.synchronize(self.dev)      # the sums are zero before any stream adds to them
        if self.learned and self.check0 is not None and len(self.check0):
            self.cfast.add(self.check0)
            self.csafe.add(self.check0)
            self.n_check = len(self.check0)

    def _queue_check(self):
        """Queues the check error of the sums so far on the current stream (no host synchronisation)."""
        torch = self.torch
        a, ref = self.chk
        sel = ref > 1e-3 * ref.max()
        zero = torch.zeros((), dtype=ref.dtype, device=ref.device)
        num = torch.linalg.norm(torch.where(sel, a - ref, zero))
        den = torch.linalg.norm(torch.where(sel, ref, zero))
        host = self._hosts[self._next_host]
        self._next_host = (self._next_host + 1) % len(self._hosts)
        host.copy_(torch.stack([num, den]), non_blocking=True)
        ev = torch.cuda.Event()
        ev.record()
        self._pending.append((ev, host))

    def _resolve(self, stream, keep=0):
        """Reads the queued checks but the `keep` newest, oldest first; above the tolerance, falls back
        (the checks still queued then no longer matter)."""
        while len(self._pending) > keep:
            ev, host = self._pending.pop(0)
            ev.synchronize()
            num, den = float(host[0]), float(host[1])
            e = num / den if den > 0. else float('inf')
            self.check_errors.append(e)
            if e > self.tol:
                self._pending = []
                self._fall_back(stream)
                return

    def _fall_back(self, stream):
        self.fell_back = True
        self.acc.zero_()                               # on `stream` (the caller's context)
        for b in self.added_fast:
            self.safe.add(b, stream)
            self.rerun += len(b)
        self.added_fast = []

    def _ctx(self, stream):
        torch = self.torch
        return torch.cuda.stream(torch.cuda.ExternalStream(stream, device=self.dev))

    def add(self, offsets, stream=None):
        """Adds the electrons (offsets as MultiE.add) in batches of max_batch, each with its check.
        `stream`: a CUDA stream handle (default: the object's own stream); the checks' reductions run
        on it too.  The work is queued, not waited for: ``mean()`` waits."""
        from .multie import offset_array
        off = offset_array(offsets)
        stream = stream or self._stream.cuda_stream
        with self._ctx(stream):
            for i0 in range(0, len(off), self.max_batch):
                b = off[i0:i0 + self.max_batch]
                # the check of the batch before last (queued behind that batch) is read: the host
                # then plans this batch while the device still runs the last one
                if self.learned and not self.fell_back:
                    self._resolve(stream, keep=1)
                if self.learned and not self.fell_back:
                    # the batch first (the device starts on it while the host plans the check
                    # electrons), then its check electron at both factors and the check
                    self.fast.add(b, stream)
                    self.added_fast.append(b)
                    self.cfast.add(b[:1], stream)
                    self.csafe.add(b[:1], stream)
                    self.n_check += 1
                    self._queue_check()
                else:
                    self.safe.add(b, stream)
                self.batches += 1
                self.n += len(b)

    def resolve(self, stream=None):
        """Reads the queued checks (falling back if one fails); mean() calls it."""
        stream = stream or self._stream.cuda_stream
        with self._ctx(stream):
            self._resolve(stream)

    @property
    def fallbacks(self):
        return int(self.fell_back)

    def mean(self, stream=None):
        self.resolve(stream)
        self.torch.cuda.synchronize(self.dev)
        return (self.acc / max(self.n, 1)).cpu().numpy()

    def reset(self):
        """Clears the accumulated intensity, the check sums (the construction-time check set is
        propagated again) and the counters; plans and captured graphs are kept."""
        self.torch.cuda.synchronize(self.dev)
        self.acc.zero_()
        for m in (self.fast, self.safe, self.cfast, self.csafe):
            if m is not None:
                m.reset()
        self._start()


# ------------------------------------------------------------------------------------------------
# training
# ------------------------------------------------------------------------------------------------
def make_data(n_samples, seed, dev, threads=8, log=print, path=None, chunk=2000):
    """Features, targets, label errors and evaluation counts of n_samples seeded cases, labelled on
    `threads` host threads (each with its own CUDA stream: the planner runs on the host).  A case
    whose labelling fails (no usable reference intensity) is replaced by the next seed.  With `path`
    the data so far is saved after every `chunk` samples, and a run resumes from a saved file."""
    import torch
    from concurrent.futures import ThreadPoolExecutor
    X = np.zeros((n_samples, N_IN), np.float32)
    T = np.zeros((n_samples, N_OUT), np.float32)
    E = np.zeros(n_samples)
    NE = np.zeros(n_samples, np.int32)
    done0 = 0
    if path and os.path.exists(path):
        d = np.load(path)
        done0 = min(len(d['X']), n_samples)
        X[:done0], T[:done0], E[:done0], NE[:done0] = d['X'][:done0], d['T'][:done0], d['E'][:done0], d['NE'][:done0]
        log('resuming after %d saved samples' % done0)
    t0 = time.time()
    local = threading.local()

    def one(s):
        if not hasattr(local, 'stream'):
            local.stream = torch.cuda.Stream(dev)
        for attempt in range(20):
            rng = np.random.default_rng([seed, s, attempt])
            case = sample_case(rng)
            try:
                with torch.cuda.stream(local.stream):
                    x = case_features(case, dev).cpu().numpy()
                    lab, e, ne = label_case(case, dev, local.stream)
            except ValueError:
                continue
            X[s], T[s], E[s], NE[s] = x, target(lab), e, ne
            return
        raise RuntimeError('no usable case for sample %d' % s)

    with ThreadPoolExecutor(threads) as ex:
        for c0 in range(done0, n_samples, chunk):
            c1 = min(n_samples, c0 + chunk)
            list(ex.map(one, range(c0, c1)))
            torch.cuda.synchronize(dev)
            torch.cuda.empty_cache()           # the threads' streams each keep freed blocks otherwise
            log('labelled %d (%.0f s)' % (c1, time.time() - t0))
            if path:
                np.savez_compressed(path, X=X[:c1], T=T[:c1], E=E[:c1], NE=NE[:c1])
    return X, T, E, NE


def main():
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument('--samples', type=int, default=20000)
    ap.add_argument('--val', type=float, default=0.1)
    ap.add_argument('--epochs', type=int, default=200)
    ap.add_argument('--seed', type=int, default=0)
    ap.add_argument('--threads', type=int, default=8)
    ap.add_argument('--out', default=DEFAULT_MODEL)
    ap.add_argument('--data', default=None, help='npz with features/targets to reuse or to write')
    args = ap.parse_args()
    dev = torch.device('cuda', 0)
    t0 = time.time()
    X, T, E, NE = make_data(args.samples, args.seed, dev, args.threads, path=args.data)
    t_data = time.time() - t0
    nv = int(len(X) * args.val)
    Xt, Tt = torch.from_numpy(X[nv:]).to(dev), torch.from_numpy(T[nv:]).to(dev)
    Xv, Tv = torch.from_numpy(X[:nv]).to(dev), torch.from_numpy(T[:nv]).to(dev)
    m = ResizeMLP(device=0, seed=args.seed)
    hist = m.train(Xt, Tt, Xv, Tv, epochs=args.epochs, log=print)
    # validation: chosen factors vs labels, cost relative to the conservative factors (cost model)
    pred = m.predict(Xv).cpu().numpy()
    cost_pred = cost_label = 0.
    at_least_label = 0
    for i in range(nv):
        n = int(round(2. ** float(X[i, N_IMG + 11])))
        fac = choose_grid(pred[i], n, n)
        lab = tuple(float(v) for v in 2. ** T[i])
        c2 = grid_cost(n, n, CONSERVATIVE)
        cost_pred += grid_cost(n, n, fac) / c2
        cost_label += grid_cost(n, n, lab) / c2
        at_least_label += all(new_length(n, fac[2 * a], fac[2 * a + 1]) >= new_length(n, lab[2 * a], lab[2 * a + 1])
                              for a in (0, 1))
    meta = dict(samples=int(len(X)), val=int(nv), epochs=int(args.epochs), final_train=float(hist[-1][1]),
                final_val=float(hist[-1][2]), val_grid_at_least_label=float(at_least_label) / max(nv, 1),
                val_cost_pred=float(cost_pred) / max(nv, 1), val_cost_label=float(cost_label) / max(nv, 1),
                labels_conservative=float(np.mean(np.all(np.abs(T - 1.) < 1e-6, axis=1))),
                mean_evaluations_per_label=float(np.mean(NE)), cost_conservative=1.0,
                cost_model='grid_cost: autotuned per-length pass times, relative to the conservative factors',
                tol=TOL_LABEL, axis_tol=AXIS_TOL, grid_range=GRID_R.tolist(), grid_resolution=GRID_D.tolist(),
                seconds_data=float(t_data), seconds=float(time.time() - t0))
    m.save(args.out, meta)
    print(json.dumps(meta))


if __name__ == '__main__':
    main()
