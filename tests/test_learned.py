"""Learned resize factors: the MLP kernels against the FP64 oracle (forward, gradients, Adam),
the feature kernels, training, and what the trained network gains over fixed conservative factors."""
import math
import os
import sys

import numpy as np
import pytest

from tests.helpers import REPO

sys.path.insert(0, os.path.join(REPO, 'oracle'))
import mlp_oracle as MO  # noqa: E402  (the checker)

from srw_b200 import learned  # noqa: E402


def test_oracle_gradients_match_central_differences():
    rng = np.random.default_rng(0)
    sizes = [7, 5, 4, 2]
    Ws = [rng.standard_normal((a, c)) * 0.5 for a, c in zip(sizes[:-1], sizes[1:])]
    bs = [rng.standard_normal(c) * 0.1 for c in sizes[1:]]
    X = rng.standard_normal((6, 7))
    T = rng.standard_normal((6, 2))
    out, Z, Y = MO.forward(X, Ws, bs)
    dW, _ = MO.backward(MO.mse(out, T)[1], Ws, Z, Y)
    for l, idx in ((0, (3, 2)), (1, (0, 1)), (2, (3, 1))):
        assert abs(MO.numeric_grad(X, T, Ws, bs, l, idx) - dW[l][idx]) < 1e-7


def test_targets_and_grid_choice():
    assert np.allclose(2. ** learned.target((1.25, 2.0, 0.5, 1.0)), [1.25, 2.0, 0.5, 1.0])
    C = learned.CONSERVATIVE
    assert learned.new_length(1024, 1., 1.) == 1024 and learned.new_length(1024, 2., 2.) == 4096
    assert learned.new_length(1024, 1.25, 1.75) == 2240 and learned.new_length(1000, 1.0001, 1.) == 1000
    rng = np.random.default_rng(0)
    for _ in range(200):
        pred = rng.uniform(-1.2, 1.2, 4)
        n = int(rng.choice([256, 512, 1024]))
        fac = learned.choose_grid(pred, n, n)
        if np.all(2. ** pred <= 2.):
            # every factor at or above the prediction, and no dearer than the conservative factors
            assert all(f >= 2. ** p - 1e-6 for f, p in zip(fac, pred)), (pred, fac)
            assert learned.grid_cost(n, n, fac) <= learned.grid_cost(n, n, C) * (1 + 1e-12)
        else:
            assert all(f in learned.GRID_R or f in learned.GRID_D for f in fac)
    # the cheapest choice for a prediction at the grid's floor is the floor itself
    assert learned.choose_grid(np.log2([0.5, 1., 0.5, 1.]), 1024, 1024) == (0.5, 1., 0.5, 1.)
    assert learned.grid_cost(1024, 1024, (1., 1.25, 1., 1.25)) < learned.grid_cost(1024, 1024, C)


# ------------------------------------------------------------------------------------------------
# GPU
# ------------------------------------------------------------------------------------------------
def _torch():
    torch = pytest.importorskip('torch')
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    return torch


@pytest.mark.gpu
def test_gemm_all_transposes():
    torch = _torch()
    from srw_b200 import capi
    import ctypes as C
    rng = np.random.default_rng(1)
    M, N, K = 70, 130, 33
    for ta in (0, 1):
        for tb in (0, 1):
            A = rng.standard_normal((K, M) if ta else (M, K)).astype(np.float32)
            B = rng.standard_normal((N, K) if tb else (K, N)).astype(np.float32)
            Cm = rng.standard_normal((M, N)).astype(np.float32)
            dA, dB, dC = (torch.from_numpy(a).cuda() for a in (A, B, Cm))
            r = capi.lib().srwgMlpGemm(M, N, K, dA.data_ptr(), A.shape[1], ta, dB.data_ptr(), B.shape[1], tb,
                                       dC.data_ptr(), N, 0.5, 2.0, None)
            assert r == 0
            want = 0.5 * ((A.T if ta else A).astype(np.float64) @ (B.T if tb else B).astype(np.float64)) + 2.0 * Cm
            np.testing.assert_allclose(dC.cpu().numpy(), want, rtol=1e-4, atol=1e-4)


@pytest.mark.gpu
def test_mlp_forward_backward_vs_fp64_oracle():
    """Gradients of the CUDA kernels against the FP64 oracle's analytic (and numerically checked)
    gradients: relative error below 1e-4."""
    torch = _torch()
    m = learned.ResizeMLP(n_in=40, hidden=(32, 24), n_out=2, seed=3)
    rng = np.random.default_rng(4)
    X = rng.standard_normal((50, 40)).astype(np.float32)
    T = rng.standard_normal((50, 2)).astype(np.float32)
    dX, dT = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
    out = m.forward(dX)
    loss, dout = m.loss_grad(out, dT)
    dW, db = m.backward(dout)
    torch.cuda.synchronize()
    Ws = [w.cpu().numpy() for w in m.W]
    bs = [b.cpu().numpy() for b in m.b]
    o, Z, Y = MO.forward(X, Ws, bs)
    l, g = MO.mse(o, T)
    rW, rb = MO.backward(g, Ws, Z, Y)
    assert np.linalg.norm(out.cpu().numpy() - o) / np.linalg.norm(o) < 1e-5
    assert abs(float(loss.item()) - l) / l < 1e-5
    for a, b in zip(dW + db, rW + rb):
        a = a.cpu().numpy()
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-4


@pytest.mark.gpu
def test_adam_step_matches_formula():
    torch = _torch()
    m = learned.ResizeMLP(n_in=5, hidden=(4,), n_out=1, seed=0)
    w0 = m.W[0].cpu().numpy().astype(np.float64)
    g = [torch.full_like(w, 0.5) for w in m.W]
    gb = [torch.full_like(b, -0.25) for b in m.b]
    m.adam(g, gb, lr=0.01)
    m.adam(g, gb, lr=0.01)
    torch.cuda.synchronize()
    mm, vv, w = 0., 0., w0.copy()
    for t in (1, 2):
        mm = 0.9 * mm + 0.1 * 0.5
        vv = 0.999 * vv + 0.001 * 0.25
        w = w - 0.01 * (mm / (1 - 0.9 ** t)) / (math.sqrt(vv / (1 - 0.999 ** t)) + 1e-8)
    np.testing.assert_allclose(m.W[0].cpu().numpy(), w, rtol=1e-5, atol=1e-6)


@pytest.mark.gpu
def test_features_downsample_and_curvature():
    torch = _torch()
    n, r, E, R = 256, 1e-3, 5000., 12.0
    lam = 1.239842e-06 / E
    x = np.linspace(-r, r, n)
    X, Y = np.meshgrid(x, x)
    ex = (np.exp(-(X * X + Y * Y) / (2 * (0.3e-3) ** 2)) * np.exp(1j * math.pi * (X * X + Y * Y) / (lam * R))).astype(
        np.complex64)
    ey = (0.1 * ex).astype(np.complex64)
    mesh = dict(nx=n, ny=n, xStart=-r, xFin=r, yStart=-r, yFin=r)
    # the wavefront's own radius is 5 % off: the fit recovers the rest from the (resolved) residual phase
    f = learned.features(torch.from_numpy(ex).cuda(), torch.from_numpy(ey).cuda(), mesh, E, ('c', 1e-3, 1e-3), 10.,
                         10., torch.device('cuda', 0), Rx=1.05 * R, Ry=0.95 * R).cpu().numpy()
    I = np.abs(ex.astype(np.complex128)) ** 2 + np.abs(ey.astype(np.complex128)) ** 2
    d = MO.downsample64(I)
    np.testing.assert_allclose(f[:4096], np.sqrt(d / d.max()).ravel(), rtol=1e-5, atol=1e-6)
    assert abs(f[4096] * R - 1.) < 0.01 and abs(f[4097] * R - 1.) < 0.01      # fitted 1/R


@pytest.mark.gpu
def test_training_fits_a_smooth_map():
    torch = _torch()
    rng = np.random.default_rng(5)
    X = rng.standard_normal((600, 12)).astype(np.float32)
    T = np.stack([np.tanh(X[:, 0] + 0.5 * X[:, 1]), 0.3 * X[:, 2] * X[:, 3]], 1).astype(np.float32)
    m = learned.ResizeMLP(n_in=12, hidden=(64, 64), n_out=2, seed=1)
    h = m.train(torch.from_numpy(X[:500]).cuda(), torch.from_numpy(T[:500]).cuda(),
                torch.from_numpy(X[500:]).cuda(), torch.from_numpy(T[500:]).cuda(), epochs=60, batch=50, lr=3e-3)
    assert h[-1][1] < 0.1 * h[0][1]
    assert h[-1][2] < 0.3 * float(np.mean(T[500:] ** 2))


@pytest.mark.gpu
def test_trained_model_gain_over_conservative_factors():
    """Held-out wavefronts (a seed not used in training): the trained network's factors (with the
    run-time check against the conservative factors and its fallback) against the oversampled
    propagation, and the measured propagation time (CUDA events) against the conservative factors
    (2, 2, 2, 2): a real gain (> 1) at a median error below the 1e-3 tolerance."""
    torch = _torch()
    if not os.path.exists(learned.DEFAULT_MODEL):
        pytest.skip('no trained model in the package')
    m = learned.ResizeMLP.load(learned.DEFAULT_MODEL)
    if m.sizes[0] != learned.N_IN or m.sizes[-1] != learned.N_OUT:
        pytest.skip('packaged model was trained for other features')
    dev = torch.device('cuda', 0)
    rng = np.random.default_rng(123456)
    t_fac, t_con, errs, n_fallback = 0., 0., [], 0

    def timed(case, fac):
        # the propagation's device time: planned once, field resident, the passes' CUDA-event times
        # (no host gaps between launches) summed, best of three executions
        from srw_b200 import srwlib as mod
        from srw_b200.plan import Plan
        p = Plan(learned._wfr(mod, case),
                 learned.beamline(mod, case['ap'], case['f'], case['L'], fac, case.get('drift_mode', 4)), device=0)
        ex, ey = torch.from_numpy(case['ex']).to(dev), torch.from_numpy(case['ey']).to(dev)
        ox, oy = p.new_output()
        p.execute(ex, ey, ox, oy)                                       # warm-up
        torch.cuda.synchronize()
        t = min(sum(p.execute_timed(ex, ey, ox, oy)) for _ in range(3))
        I, om = learned.propagate_intensity(case, fac, dev)
        return I, om, t

    for _ in range(16):
        case = learned.sample_case(rng)
        fac, fb, _ = learned.choose_factors(m, case, dev)
        n_fallback += fb
        rf = learned.ref_factors(case['mesh']['nx'])
        Iref, omref = learned.propagate_intensity(case, rf + rf, dev)
        I, om, tf = timed(case, fac)
        _, _, tc = timed(case, learned.CONSERVATIVE)
        errs.append(learned.factor_error(I, om, Iref, omref, learned.eval_box(Iref, omref)))
        t_fac += tf
        t_con += tc
    gain = t_con / t_fac
    print('measured gain over conservative factors %.2f, fallbacks %d, median error %.2e' %
          (gain, n_fallback, np.median(errs)))
    if os.environ.get('SRWG_TEST_REPORT'):
        import json
        with open(os.environ['SRWG_TEST_REPORT'], 'a') as f:
            f.write(json.dumps({"test": "learned_gain", "cases": 16, "gain_device_time": gain,
                                "fallbacks": int(n_fallback), "median_rel_err": float(np.median(errs))}) + '\n')
    assert gain > 1.0
    assert np.median(errs) < 1e-3


@pytest.mark.gpu
def test_checked_multie_falls_back_and_rebuilds():
    """learned.CheckedMultiE: a check that every batch meets gives the learned factors' mean
    intensity, its errors those of the check set's two mean intensities; a check that fails at the
    first batch gives the conservative factors' mean (the first batch and the one queued after it,
    both run before the check was read, are propagated again); a check that fails after two batches
    propagates those two again with the conservative factors, so the result is again the
    conservative factors' mean of all electrons (same batches, FP64 sums)."""
    torch = _torch()
    from srw_b200 import srwlib as mod
    from srw_b200.multie import MultiE, sample_offsets
    dev = torch.device('cuda', 0)
    case = learned.sample_case(np.random.default_rng(7), n=256)
    w = learned._wfr(mod, case)
    mk = lambda f: learned.beamline(mod, case['ap'], case['f'], case['L'], f)  # noqa: E731
    fac = (1.25, 1.5, 1.25, 1.5)
    from srw_b200.plan import Plan
    om = Plan(w, mk(learned.CONSERVATIVE), device=0).output_mesh()
    acc = dict(nx=128, ny=128, xStart=om['xStart'], xFin=om['xFin'], yStart=om['yStart'], yFin=om['yFin'])
    offs = sample_offsets(24, 20e-6, 5e-6, 5e-6, 2e-6, seed=3, sig_e=1e-3)
    chk = sample_offsets(4, 20e-6, 5e-6, 5e-6, 2e-6, seed=4, sig_e=1e-3)

    def plain(f):
        me = MultiE(w, mk(f), acc, max_batch=8, graph=False, device=0)
        me.add(offs)
        return me.mean()

    m_cons, m_fast = plain(learned.CONSERVATIVE), plain(fac)
    kw = dict(max_batch=8, safe_batch=8, graph=False, device=0, check_offsets=chk)
    ok = learned.CheckedMultiE(w, mk, fac, acc, tol=1.0, **kw)
    ok.add(offs)
    np.testing.assert_allclose(ok.mean(), m_fast, rtol=1e-12, atol=0)
    assert not ok.fell_back and ok.n_check == 4 + 3 and len(ok.check_errors) == 3
    Ia = learned.mean_intensity(case, fac, np.vstack([chk, offs[0:1], offs[8:9], offs[16:17]]), acc, dev)
    Ib = learned.mean_intensity(case, learned.CONSERVATIVE, np.vstack([chk, offs[0:1], offs[8:9], offs[16:17]]), acc,
                                dev)
    assert abs(ok.check_errors[-1] - learned.rel_err(Ia, Ib)) <= 1e-9 * max(1e-12, learned.rel_err(Ia, Ib))
    first = learned.CheckedMultiE(w, mk, fac, acc, tol=-1.0, **kw)
    first.add(offs)
    np.testing.assert_allclose(first.mean(), m_cons, rtol=1e-12, atol=0)
    assert first.fell_back and first.rerun == 16 and len(first.check_errors) == 1
    late = learned.CheckedMultiE(w, mk, fac, acc, tol=1.0, **kw)
    late.add(offs[:16])
    late.tol = -1.0
    late.add(offs[16:])
    np.testing.assert_allclose(late.mean(), m_cons, rtol=1e-12, atol=0)
    assert late.fell_back and late.rerun == 16
    # a checked batch of 8 run as launches of 4: the same electrons and checks, the sums in another order
    split = learned.CheckedMultiE(w, mk, fac, acc, tol=1.0, launch_batch=4, **kw)
    split.add(offs)
    np.testing.assert_allclose(split.mean(), m_fast, rtol=1e-10, atol=0)
    assert not split.fell_back and len(split.check_errors) == 3
    np.testing.assert_allclose(split.check_errors, ok.check_errors, rtol=1e-12)
    split_fb = learned.CheckedMultiE(w, mk, fac, acc, tol=-1.0, launch_batch=4, **kw)
    split_fb.add(offs)
    np.testing.assert_allclose(split_fb.mean(), m_cons, rtol=1e-12, atol=0)
    assert split_fb.fell_back and split_fb.rerun == 16
    assert np.linalg.norm(m_fast - m_cons) > 0
