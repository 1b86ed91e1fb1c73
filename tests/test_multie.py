"""Partially coherent (multi-electron) propagation: electron sampling and sharding, the mean-intensity
accumulation (avg_update_interp order 1), the sum over ranks (gloo, 2 processes on the CPU), and on
the GPU the batched C-ABI path (srwgMultiE*) against the FP64 oracle run electron by electron."""
import os
import sys

import numpy as np
import pytest

from srw_b200.multie import sample_offsets, shard
from tests.golden_cases import case_io, load
from tests.helpers import O, beamline, make_wfr, rel_l2

TOL = 1e-4                       # relative L2 of the mean intensity, FP32 GPU path vs FP64 oracle
SIG = (30e-6, 5e-6, 5e-6, 2e-6)  # source phase space: sigma x [m], x' [rad], y [m], y' [rad]
D, INDEX = load()


def base_case():
    c = next(c for c in INDEX if c['name'] == 'c1_64')
    i, o = case_io(D, 'c1_64')
    sc = dict(Rx=i['Rx'], Ry=i['Ry'], dRx=i['dRx'], dRy=i['dRy'], xc=i['xc'], yc=i['yc'])
    acc = dict(nx=96, ny=80, xStart=0.8 * o['mesh']['xStart'], xFin=0.8 * o['mesh']['xFin'],
               yStart=0.8 * o['mesh']['yStart'], yFin=0.8 * o['mesh']['yFin'], eStart=i['mesh']['eStart'])
    return i, sc, c['elements'], c['props'], acc


def oracle_sum(i, sc, elements, props, acc, offsets):
    """FP64 oracle: the reference's per-electron loop (offset, propagate, intensity, interpolate)."""
    s = np.zeros((acc['ny'], acc['nx']))
    for off in offsets:
        ex, ey, mesh, sc2 = O.electron_offset(i['ex'], i['ey'], i['mesh'], sc, *off)
        w = O.Wfr.from_srwl(ex, ey, mesh, sc2['Rx'], sc2['Ry'], sc2['dRx'], sc2['dRy'], sc2['xc'], sc2['yc'])
        O.propagate(w, [tuple(e) for e in elements], props)
        O.add_interp_bilinear(s, acc, O.total_intensity(w.ex, w.ey), w.out_mesh())
    return s


def test_offsets_counter_based_and_shards():
    a = sample_offsets(10, *SIG, seed=7)
    b = np.concatenate([sample_offsets(4, *SIG, seed=7), sample_offsets(6, *SIG, seed=7, first=4)])
    assert np.array_equal(a, b)
    assert abs(np.std(sample_offsets(4000, *SIG, seed=1)[:, 0]) / SIG[0] - 1.) < 0.05
    parts = [shard(103, r, 4) for r in range(4)]
    allk = np.sort(np.concatenate(parts))
    assert np.array_equal(allk, np.arange(103))
    assert max(len(p) for p in parts) - min(len(p) for p in parts) <= 1


def test_interp_matches_reference_loop():
    """The vectorised accumulation against a scalar restatement of avg_update_interp (order 1)."""
    rng = np.random.default_rng(3)
    I = rng.random((7, 9)).astype(np.float32)
    mesh = dict(nx=9, ny=7, xStart=-1.0, xFin=1.2, yStart=-0.7, yFin=0.9)
    acc_mesh = dict(nx=11, ny=6, xStart=-1.3, xFin=1.4, yStart=-0.9, yFin=1.0)
    got = O.add_interp_bilinear(np.zeros((6, 11)), acc_mesh, I, mesh)
    xs, ys = (mesh['xFin'] - mesh['xStart']) / 8, (mesh['yFin'] - mesh['yStart']) / 6
    want = np.zeros((6, 11))
    for iy in range(6):
        y = acc_mesh['yStart'] + iy * (acc_mesh['yFin'] - acc_mesh['yStart']) / 5
        for ix in range(11):
            x = acc_mesh['xStart'] + ix * (acc_mesh['xFin'] - acc_mesh['xStart']) / 10
            ix0 = int(np.trunc((x - mesh['xStart']) / xs + 1.e-09))
            iy0 = int(np.trunc((y - mesh['yStart']) / ys + 1.e-09))
            if ix0 < 0 or ix0 >= 8 or iy0 < 0 or iy0 >= 6:
                continue
            tx = (x - (mesh['xStart'] + xs * ix0)) / xs
            ty = (y - (mesh['yStart'] + ys * iy0)) / ys
            a00, f10, f01, f11 = (float(I[iy0, ix0]), float(I[iy0, ix0 + 1]), float(I[iy0 + 1, ix0]),
                                  float(I[iy0 + 1, ix0 + 1]))
            want[iy, ix] = a00 + tx * ((f10 - a00) + ty * (a00 - f01 - f10 + f11)) + ty * (f01 - a00)
    np.testing.assert_allclose(got, want, rtol=1e-14, atol=1e-14)


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    import torch
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        from srw_b200.multie import allreduce_mean, shard_offsets
        i, sc, el, pp, acc = base_case()
        n = 7
        mine = shard_offsets(n, rank, world, *SIG, seed=11, sig_e=1e-3)
        # this rank's FP64 intensity sum (the oracle's per-electron loop stands in for the device
        # accumulator, which needs a GPU), reduced over the ranks by the library's own function
        part = torch.from_numpy(oracle_sum(i, sc, el, pp, acc, mine))
        mean, n_all = allreduce_mean(part, len(mine))
        if rank == 0:
            q.put((mean.numpy(), n_all, oracle_sum(i, sc, el, pp, acc, sample_offsets(n, *SIG, seed=11, sig_e=1e-3)) / n))
    finally:
        dist.destroy_process_group()


def test_sharded_sum_over_ranks_gloo():
    """Electrons sharded round-robin over 2 ranks, partial FP64 sums reduced over gloo: the mean
    equals the single-process mean."""
    import multiprocessing as mp
    import socket
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        port = s.getsockname()[1]
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    got, n_all, want = q.get(timeout=300)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert n_all == 7
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12 * np.abs(want).max())


def test_shard_offsets_union_and_offset_arrays():
    """Per-rank offsets (counter-based) add up to the single-process set; flat offset arrays need
    their column count."""
    from srw_b200.multie import offset_array, shard_offsets
    full = sample_offsets(11, *SIG, seed=4, sig_e=1e-3)
    got = np.zeros_like(full)
    for r in range(3):
        got[shard(11, r, 3)] = shard_offsets(11, r, 3, *SIG, seed=4, sig_e=1e-3)
    assert np.array_equal(got, full)
    one = full[0]
    assert offset_array(one, ncols=5).shape == (1, 5)
    assert offset_array(full[:1]).shape == (1, 5)
    assert offset_array(full[:4, :4].ravel(), ncols=4).shape == (4, 4)
    for bad in (dict(offsets=one), dict(offsets=np.zeros(20)), dict(offsets=np.zeros(20), ncols=3),
                dict(offsets=full, ncols=4), dict(offsets=np.zeros(7), ncols=5)):
        with pytest.raises(ValueError):
            offset_array(**bad)


# ------------------------------------------------------------------------------------------------
# GPU
# ------------------------------------------------------------------------------------------------
def _gpu():
    torch = pytest.importorskip('torch')
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')


def _multie(batch, graph, offsets):
    from srw_b200.multie import MultiE
    i, sc, el, pp, acc = base_case()
    w = make_wfr(i['ex'], i['ey'], i['mesh'], **sc)
    me = MultiE(w, beamline(el, pp), acc, max_batch=batch, graph=graph)
    me.add(offsets)
    return me.mean(), me.count()


@pytest.mark.gpu
def test_multie_vs_oracle():
    _gpu()
    offs = sample_offsets(6, *SIG, seed=5)
    got, n = _multie(4, False, offs)
    i, sc, el, pp, acc = base_case()
    want = oracle_sum(i, sc, el, pp, acc, offs) / 6
    assert n == 6
    assert np.abs(want).max() > 0
    assert rel_l2(got, want) < TOL


@pytest.mark.gpu
def test_multie_batch_sizes_and_graph_agree():
    _gpu()
    offs = sample_offsets(9, *SIG, seed=9)
    ref, _ = _multie(1, False, offs)
    for batch, graph in ((4, False), (4, True), (9, True)):
        got, n = _multie(batch, graph, offs)
        assert n == 9
        np.testing.assert_allclose(got, ref, rtol=1e-10, atol=1e-12 * np.abs(ref).max())


@pytest.mark.gpu
def test_multie_energy_spread_vs_oracle():
    """Electrons with a relative energy deviation (fifth offset): each wavefront's photon energy is
    rescaled to E (1 + 2 d); against the oracle loop, and visibly different from no spread."""
    _gpu()
    offs = sample_offsets(6, *SIG, seed=5, sig_e=5e-3)
    assert offs.shape == (6, 5) and np.array_equal(offs[:, :4], sample_offsets(6, *SIG, seed=5))
    got, n = _multie(4, True, offs)
    i, sc, el, pp, acc = base_case()
    want = oracle_sum(i, sc, el, pp, acc, offs) / 6
    assert n == 6
    assert rel_l2(got, want) < TOL
    flat = oracle_sum(i, sc, el, pp, acc, offs[:, :4]) / 6
    assert rel_l2(flat, want) > 10 * TOL


@pytest.mark.gpu
def test_multie_intensity_pass_vs_oracle():
    """Electrons on a grid of a specialised length (128^2 -> 320^2): the last pass transforms both
    components per CTA and writes the total intensity in column blocks (the accumulation reads one
    float per sample), its output factors folded into one scale; the mean against the oracle's
    electron-by-electron loop."""
    _gpu()
    import ctypes as C
    from srw_b200 import capi
    from srw_b200.multie import MultiE
    from tests.helpers import C1, PP, gaussian
    fam = C.c_int()
    assert capi.lib().srwgTuneGetFamily(1, 320, C.byref(fam)) == 0 and fam.value == 3
    ex, _, mesh = gaussian(128, E=2012., sig=0.35e-3, r=1.5e-3, R=20.)
    ey = 0.05j * ex
    sc = dict(Rx=20., Ry=20., dRx=0.2, dRy=0.2, xc=0., yc=0.)
    pp = [PP(), PP(0, 1.25, 2., 1.25, 2.), PP(4)]
    o = O.Wfr.from_srwl(ex, ey, mesh, 20., 20., 0.2, 0.2, 0., 0.)
    O.propagate(o, [tuple(e) for e in C1], pp)
    m = o.out_mesh()
    assert (m['nx'], m['ny']) == (320, 320)
    acc = dict(nx=96, ny=80, xStart=0.6 * m['xStart'], xFin=0.6 * m['xFin'], yStart=0.6 * m['yStart'],
               yFin=0.6 * m['yFin'], eStart=mesh['eStart'])
    offs = sample_offsets(6, *SIG, seed=21, sig_e=1e-3)
    w = make_wfr(ex, ey, mesh, **sc)
    me = MultiE(w, beamline(C1, pp), acc, max_batch=4, graph=True)
    # the to-waist output factors have one magnitude: applied as a scale of the intensity
    assert 'intensity flat' in me.describe().splitlines()[-1]
    me.add(offs)
    got = me.mean()
    want = oracle_sum(dict(ex=ex, ey=ey, mesh=mesh), sc, C1, pp, acc, offs) / 6
    assert np.abs(want).max() > 0
    assert rel_l2(got, want) < TOL


@pytest.mark.gpu
def test_multie_timed_batch_and_info():
    """srwgMultiEAddTimed runs one batch with CUDA events around every pass (the electrons are added
    as by srwgMultiEAdd: the same mean); srwgMultiEInfo lists the batch's passes as the plan API does
    and tells whether the last one writes the intensity."""
    _gpu()
    from srw_b200.multie import MultiE
    from srw_b200.plan import Plan
    i, sc, el, pp, acc = base_case()
    w = make_wfr(i['ex'], i['ey'], i['mesh'], **sc)
    offs = sample_offsets(4, *SIG, seed=31, sig_e=1e-3)
    a = MultiE(w, beamline(el, pp), acc, max_batch=4, graph=False)
    ks, inten = a.info()
    assert [k[0] for k in ks] == [k[0] for k in Plan(w, beamline(el, pp)).kernels() if k[0] != 'moments']
    ms = a.add_timed(offs)
    assert len(ms) == len(ks) + 1 and all(v > 0 for v in ms)
    assert a.count() == 4
    b = MultiE(w, beamline(el, pp), acc, max_batch=4, graph=False)
    b.add(offs)
    np.testing.assert_array_equal(a.mean(), b.mean())
    with pytest.raises(RuntimeError):
        a.add_timed(sample_offsets(5, *SIG, seed=32, sig_e=1e-3))      # more than one batch
