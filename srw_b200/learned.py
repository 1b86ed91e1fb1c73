"""Learned resize factors for the aperture -> lens -> to-waist drift beamline.

The reference's users choose the range / resolution resize factors (pp[5..8] of the propagation
parameter lists, cpp/src/core/sroptcnt.cpp:307-316) by hand; too small factors alias, too large
ones waste memory and time (the propagated grid grows with the square of their product).  This
module learns them: a small MLP (64 x 64 downsampled intensity, fitted phase-curvature radii and
the element parameters -> log2 of the range and resolution factors applied before the lens) is
trained by the project's own CUDA kernels (srwgMlp*: GEMM, bias + GELU, their gradients, MSE, Adam)
on labels that sweeps of the plain GPU propagation produce: for every training wavefront the
cheapest factor pair whose intensity agrees with an oversampled propagation (factors 3, 3) within
TOL_LABEL on a common mesh.  At run time ``choose_factors`` rounds the prediction up to the sweep
grid and checks the result (energy outside the central part of the output window); when the check
fails, the propagation falls back to the conservative factors (2, 2).

    python -m srw_b200.learned --samples 2000 --out srw_b200/models/resize_mlp.npz   # GPU: data + training

torch provides device memory and streams only; every kernel is the library's.
"""
import argparse
import ctypes as C
import json
import math
import os
import time

import numpy as np

from . import capi

GRID = np.array([1.0, 1.25, 1.5, 1.75, 2.0])       # candidate range / resolution factors
REF_FACTORS = (3.0, 3.0)                             # the oversampled propagation the labels are compared with
CONSERVATIVE = (2.0, 2.0)                            # fallback
TOL_LABEL = 1e-3                                     # relative L2 intensity error accepted by a label
N_IMG = 64 * 64
N_EXTRA = 9
N_IN = N_IMG + N_EXTRA
HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_MODEL = os.path.join(HERE, 'models', 'resize_mlp.npz')


def _check(r, what):
    capi.check(r, what)


# ------------------------------------------------------------------------------------------------
# the network
# ------------------------------------------------------------------------------------------------
class ResizeMLP(object):
    """FP32 MLP n_in -> hidden... -> n_out, GELU between layers; weights W[l] (in x out), b[l]."""

    def __init__(self, n_in=N_IN, hidden=(256, 256, 256), n_out=2, device=0, seed=0):
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
def features(ex, ey, mesh, energy, ap_d, f, L, torch_dev, Rx=0., Ry=0.):
    """Feature vector of one wavefront (complex64 CUDA tensors [ny, nx]) and its beamline:
    64 x 64 intensity (srwgWfrFeatures) normalised to its maximum and square-rooted, the fitted
    curvature radii (as 1/R [1/m]; the wavefront's own radii Rx, Ry are removed before the fit and
    added back), photon energy, aperture / wavefront size, f, L and the number of points per line."""
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
    width = mesh['xFin'] - mesh['xStart']
    extra = torch.tensor([invRx, invRz, math.log(energy / 1000.), ap_d / width, math.log(f), math.log(L),
                          math.log(width * 1e3), math.log(L / f), math.log2(nx)], dtype=torch.float32,
                         device=torch_dev)
    return torch.cat([img, extra])


# ------------------------------------------------------------------------------------------------
# synthetic wavefronts and beamlines (Gaussian and undulator-like, 1-20 keV, drifts 1-50 m,
# f 1-30 m, apertures 0.1-2 mm)
# ------------------------------------------------------------------------------------------------
def sample_case(rng, n=None):
    if n is None:
        n = 256 if rng.random() < 0.5 else 512
    E = math.exp(rng.uniform(math.log(1000.), math.log(20000.)))
    lam = 1.239842e-06 / E
    z = math.exp(rng.uniform(math.log(5.), math.log(50.)))              # source -> first element
    if rng.random() < 0.5:
        sig0 = math.exp(rng.uniform(math.log(5e-6), math.log(60e-6)))     # waist rms
        zr = 4. * math.pi * sig0 * sig0 / lam
        sig = sig0 * math.sqrt(1. + (z / zr) ** 2)
        R = z * (1. + (zr / z) ** 2)
        r = 4. * sig
        x = np.linspace(-r, r, n)
        X, Y = np.meshgrid(x, x)
        ex = np.exp(-(X * X + Y * Y) / (4. * sig * sig)) * np.exp(1j * math.pi * (X * X + Y * Y) / (lam * R))
        kind = 'gaussian'
    else:
        nper = int(rng.integers(40, 200))
        r = z * math.sqrt(3. * lam / (nper * 0.02)) * rng.uniform(0.8, 1.6)   # ~ a few rings of the harmonic
        x = np.linspace(-r, r, n)
        X, Y = np.meshgrid(x, x)
        th2 = (X * X + Y * Y) / (z * z)
        q = th2 * nper * 0.02 / (2. * lam)                              # detuning of the first harmonic
        ex = np.sinc(q) * np.exp(-1j * math.pi * q) * np.exp(1j * math.pi * (X * X + Y * Y) / (lam * z))
        R = z
        kind = 'undulator'
    ex = (ex * 1e6).astype(np.complex64)
    ey = np.zeros_like(ex)
    mesh = dict(nx=n, ny=n, xStart=-r, xFin=r, yStart=-r, yFin=r, eStart=E, eFin=E, zStart=z)
    sc = dict(Rx=R, Ry=R, dRx=0.01 * R, dRy=0.01 * R)
    ap_d = min(2e-3, max(1e-4, 2. * r * rng.uniform(0.3, 0.9)))
    f = math.exp(rng.uniform(math.log(1.), math.log(30.)))
    L = f * math.exp(rng.uniform(-0.3, 0.3))
    L = min(50., max(1., L))
    return dict(kind=kind, ex=ex, ey=ey, mesh=mesh, sc=sc, E=E, ap_d=ap_d, f=f, L=L)


def beamline(mod, ap_d, f, L, rng_f, res_f):
    """aperture -> (resize) lens -> drift to the waist, as the undulator benchmark beamline."""
    pp = lambda anal=0, pxm=1., pxd=1.: [0, 0, 1., anal, 0, pxm, pxd, pxm, pxd, 0, 0, 0]  # noqa: E731
    return mod.SRWLOptC([mod.SRWLOptA('c', 'a', ap_d, ap_d), mod.SRWLOptL(f, f), mod.SRWLOptD(L)],
                        [pp(), pp(0, rng_f, res_f), pp(4)])


def _wfr(mod, case):
    w = mod.SRWLWfr()
    n = case['mesh']['nx']
    w.allocate(1, n, n)
    for name, fld in (('arEx', case['ex']), ('arEy', case['ey'])):
        a = np.empty(2 * fld.size, np.float32)
        a[0::2] = fld.real.ravel()
        a[1::2] = fld.imag.ravel()
        setattr(w, name, a)
    for k in ('xStart', 'xFin', 'yStart', 'yFin', 'eStart', 'eFin', 'zStart'):
        setattr(w.mesh, k, case['mesh'][k])
    w.Rx, w.Ry, w.dRx, w.dRy = case['sc']['Rx'], case['sc']['Ry'], case['sc']['dRx'], case['sc']['dRy']
    return w


def _interp_bilinear(I, om, em, torch):
    """I (torch float64 [ny, nx] on mesh om) at the points of mesh em (bilinear, zero outside)."""
    ny, nx = I.shape
    xs = (om['xFin'] - om['xStart']) / (nx - 1)
    ys = (om['yFin'] - om['yStart']) / (ny - 1)
    xa = em['xStart'] + torch.arange(em['nx'], dtype=torch.float64, device=I.device) * (em['xFin'] - em['xStart']) / (em['nx'] - 1)
    ya = em['yStart'] + torch.arange(em['ny'], dtype=torch.float64, device=I.device) * (em['yFin'] - em['yStart']) / (em['ny'] - 1)
    fx = (xa - om['xStart']) / xs
    fy = (ya - om['yStart']) / ys
    ix = torch.floor(fx).long()
    iy = torch.floor(fy).long()
    okx = (ix >= 0) & (ix < nx - 1)
    oky = (iy >= 0) & (iy < ny - 1)
    ix = ix.clamp(0, nx - 2)
    iy = iy.clamp(0, ny - 2)
    tx = (fx - ix).unsqueeze(0)
    ty = (fy - iy).unsqueeze(1)
    a = I[iy][:, ix]
    b = I[iy][:, ix + 1]
    c = I[iy + 1][:, ix]
    d = I[iy + 1][:, ix + 1]
    v = a * (1 - tx) * (1 - ty) + b * tx * (1 - ty) + c * (1 - tx) * ty + d * tx * ty
    return v * (oky.unsqueeze(1) & okx.unsqueeze(0))


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


def propagate_intensity(case, rf, df, dev):
    """Plain GPU propagation with factors (rf, df): (total intensity [ny, nx] float64 CUDA, mesh)."""
    import torch
    from . import srwlib as mod
    from .plan import Plan
    w = _wfr(mod, case)
    p = Plan(w, beamline(mod, case['ap_d'], case['f'], case['L'], rf, df), device=dev.index)
    ex = torch.from_numpy(case['ex']).to(dev)
    ey = torch.from_numpy(case['ey']).to(dev)
    ox, oy = p.new_output()
    p.execute(ex, ey, ox, oy)
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
    the oversampled reference interpolated to those nodes by cubic Lagrange interpolation (its
    finer mesh and the fourth-order interpolation keep that error well below the tolerance); 1 when
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


def label_case(case, dev):
    """Sweep of the candidate factor pairs against the oversampled propagation: returns
    (best (rf, df): the cheapest by grid_cost within TOL_LABEL, errors [len(GRID), len(GRID)])."""
    n = case['mesh']['nx']
    Iref, omref = propagate_intensity(case, *REF_FACTORS, dev)
    box = eval_box(Iref, omref)
    errs = np.full((len(GRID), len(GRID)), np.inf)
    best, best_cost = CONSERVATIVE, None
    for i, rf in enumerate(GRID):
        for j, df in enumerate(GRID):
            I, om = propagate_intensity(case, rf, df, dev)
            e = factor_error(I, om, Iref, omref, box)
            errs[i, j] = e
            cost = grid_cost(n, rf, df)
            if e <= TOL_LABEL and (best_cost is None or cost < best_cost):
                best, best_cost = (rf, df), cost
    return best, errs


def case_features(case, dev):
    import torch
    ex = torch.from_numpy(case['ex']).to(dev)
    ey = torch.from_numpy(case['ey']).to(dev)
    return features(ex, ey, case['mesh'], case['E'], case['ap_d'], case['f'], case['L'], dev, case['sc']['Rx'],
                    case['sc']['Ry'])


def target(factors):
    return np.log2(np.array(factors, np.float32))


GENERAL_COST = 5.0     # per-point time of a general-length (not power-of-two) grid relative to a power of two


def grid_cost(n, rf, df):
    """Cost model of propagating an n x n wavefront with factors (rf, df): points of the resized
    grid (round-half-up of n rf df, as RadResizeGen) times GENERAL_COST when that size is not a power
    of two (measured: the general-length passes take about five times longer per point)."""
    m = int(math.floor(n * rf * df + 0.5))
    return float(m) * m * (1. if (m & (m - 1)) == 0 else GENERAL_COST)


def choose_grid(pred, n):
    """Prediction (log2 factors) -> the cheapest grid pair (grid_cost) with both factors not below it."""
    lo = [2. ** float(v) - 1e-6 for v in pred]
    best, best_cost = (float(GRID[-1]), float(GRID[-1])), None
    for rf in GRID:
        for df in GRID:
            if rf >= lo[0] and df >= lo[1]:
                c = grid_cost(n, rf, df)
                if best_cost is None or c < best_cost:
                    best, best_cost = (float(rf), float(df)), c
    return best


def round_up(pred):
    """Prediction (log2 factors) -> the smallest grid factors not below it."""
    out = []
    for v in pred:
        f = 2. ** float(v)
        cand = GRID[GRID >= f - 1e-6]
        out.append(float(cand[0]) if len(cand) else float(GRID[-1]))
    return tuple(out)


def output_check(I):
    """Run-time check of a propagation with predicted factors: the fraction of the intensity in
    the outer eighth of the output window on each side (aliasing / clipping indicator)."""
    ny, nx = I.shape
    b = max(1, nx // 8), max(1, ny // 8)
    tot = float(I.sum())
    inner = float(I[b[1]:ny - b[1], b[0]:nx - b[0]].sum())
    return (tot - inner) / tot if tot > 0 else 1.


def choose_factors(model, case, dev, check_tol=1e-3):
    """(factors, used_fallback): the model's factors when the propagation with them passes
    output_check, else the conservative ones."""
    feat = case_features(case, dev).unsqueeze(0)
    pred = model.predict(feat)[0].cpu().numpy()
    fac = choose_grid(pred, case['mesh']['nx'])
    I, _ = propagate_intensity(case, *fac, dev)
    if output_check(I) > check_tol:
        return CONSERVATIVE, True
    return fac, False


def main():
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument('--samples', type=int, default=2000)
    ap.add_argument('--val', type=float, default=0.15)
    ap.add_argument('--epochs', type=int, default=300)
    ap.add_argument('--seed', type=int, default=0)
    ap.add_argument('--out', default=DEFAULT_MODEL)
    ap.add_argument('--data', default=None, help='npz with features/targets to reuse')
    args = ap.parse_args()
    dev = torch.device('cuda', 0)
    t0 = time.time()
    if args.data and os.path.exists(args.data):
        d = np.load(args.data)
        X, T, errs = d['X'], d['T'], d['errs']
    else:
        rng = np.random.default_rng(args.seed)
        X = np.zeros((args.samples, N_IN), np.float32)
        T = np.zeros((args.samples, 2), np.float32)
        errs = np.zeros((args.samples, len(GRID), len(GRID)))
        for s in range(args.samples):
            case = sample_case(rng)
            X[s] = case_features(case, dev).cpu().numpy()
            best, e = label_case(case, dev)
            T[s] = target(best)
            errs[s] = e
            if s % 100 == 0:
                print('sample %d (%.0f s)' % (s, time.time() - t0), flush=True)
        if args.data:
            np.savez_compressed(args.data, X=X, T=T, errs=errs)
    nv = int(len(X) * args.val)
    Xt, Tt = torch.from_numpy(X[nv:]).to(dev), torch.from_numpy(T[nv:]).to(dev)
    Xv, Tv = torch.from_numpy(X[:nv]).to(dev), torch.from_numpy(T[:nv]).to(dev)
    m = ResizeMLP(device=0, seed=args.seed)
    hist = m.train(Xt, Tt, Xv, Tv, epochs=args.epochs, log=print)
    # validation: chosen factors against the sweep errors; cost relative to the conservative factors
    pred = m.predict(Xv).cpu().numpy()
    ok, cost_pred, cost_label = 0, 0., 0.
    for i in range(nv):
        n = int(round(2. ** float(X[i, N_IMG + 8])))
        fac = choose_grid(pred[i], n)
        a, b = int(np.argmin(np.abs(GRID - fac[0]))), int(np.argmin(np.abs(GRID - fac[1])))
        ok += errs[i, a, b] <= TOL_LABEL
        c2 = grid_cost(n, *CONSERVATIVE)
        cost_pred += grid_cost(n, *fac) / c2
        lab = 2. ** T[i]
        cost_label += grid_cost(n, float(lab[0]), float(lab[1])) / c2
    meta = dict(samples=int(len(X)), val=int(nv), epochs=int(args.epochs), final_train=float(hist[-1][1]),
                final_val=float(hist[-1][2]), val_within_tol=float(ok) / max(nv, 1),
                val_cost_pred=float(cost_pred) / max(nv, 1), val_cost_label=float(cost_label) / max(nv, 1),
                cost_conservative=1.0, cost_model='grid_cost, relative to the conservative factors',
                general_cost=GENERAL_COST, tol=TOL_LABEL, seconds=float(time.time() - t0))
    m.save(args.out, meta)
    print(json.dumps(meta))


if __name__ == '__main__':
    main()
