"""Partially coherent (multi-electron) propagation on the GPU.

The reference's ``srwl_wfr_emit_prop_multi_e`` (env/python/srwpy/srwlib.py:8506) loops in Python
over macro-electrons: field, ``srwl.PropagElecField``, ``srwl.CalcIntFromElecField`` and
``SRWLStokes.avg_update_interp`` onto a common mesh.  ``MultiE`` runs that loop on the device in
batches (C-ABI ``srwgMultiE*``): electron wavefronts are the base wavefront offset as
``SRWLWfr.sim_src_offset`` does (srwlib.py:2803), every pass of the beamline is one launch per
batch, and the intensities are summed in FP64 on the device.

    me = MultiE(base_wfr, optBL, acc_mesh, max_batch=8, graph=True)
    me.add(offsets)                 # [n, 4] float64: x [m], x' [rad], y [m], y' [rad]
    mean = me.mean()                # [ny, nx] float64 mean intensity on acc_mesh

``sample_offsets`` draws the offsets from an uncorrelated Gaussian source phase space with a
counter-based generator (numpy Philox), so any subset of electrons can be drawn independently,
e.g. one shard per rank (``shard``).
"""
import ctypes as C

import numpy as np

from . import capi
from .srwlpy import make_c_optc, make_c_wfr


def sample_offsets(n, sig_x, sig_xp, sig_y, sig_yp, seed=0, first=0, sig_e=None):
    """Offsets of electrons first .. first+n-1: [n, 4] = (x, x', y, y'), independent normals, and with
    sig_e a fifth column, the relative energy deviation.  Electron k always gets the same numbers
    (Philox stream keyed by the seed, advanced to k; the first four do not depend on sig_e)."""
    m = 4 if sig_e is None else 5
    out = np.empty((n, m), np.float64)
    sig = np.array([sig_x, sig_xp, sig_y, sig_yp] + ([] if sig_e is None else [sig_e]), np.float64)
    for i in range(n):
        g = np.random.Generator(np.random.Philox(key=seed, counter=[first + i, 0, 0, 0]))
        out[i] = g.standard_normal(m) * sig
    return out


def shard(n_total, rank, world):
    """Electron indices of one rank: round-robin, so every rank gets the same mix of electrons."""
    return np.arange(rank, n_total, world, dtype=np.int64)


def shard_offsets(n_total, rank, world, sig_x, sig_xp, sig_y, sig_yp, seed=0, sig_e=None):
    """Offsets of this rank's electrons (``shard``) out of n_total: [len(shard), 4 or 5], electron k
    drawn exactly as ``sample_offsets`` draws it, so the union over ranks is the single-process set."""
    idx = shard(n_total, rank, world)
    m = 4 if sig_e is None else 5
    out = np.empty((len(idx), m), np.float64)
    for j, k in enumerate(idx):
        out[j] = sample_offsets(1, sig_x, sig_xp, sig_y, sig_yp, seed=seed, first=int(k), sig_e=sig_e)[0]
    return out


def allreduce_mean(acc, n_local, group=None):
    """Mean intensity over all ranks: sums the ranks' FP64 intensity accumulators (a torch tensor,
    in place; NCCL for CUDA tensors, gloo for CPU ones) and their electron counts with one
    all-reduce each, and returns (acc / n_total, n_total).  Every rank calls it, in the same order
    as its other collectives."""
    import torch
    import torch.distributed as dist
    cnt = torch.tensor([float(n_local)], dtype=torch.float64, device=acc.device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(acc, group=group)
        dist.all_reduce(cnt, group=group)
    n = int(round(float(cnt.item())))
    return (acc / n if n > 0 else acc.clone()), n


def offset_array(offsets, ncols=None):
    """Electron offsets as a contiguous [n, 4] or [n, 5] float64 array.  A 2-D array gives its own
    column count (ncols, when given, must agree); a flat array is split into rows of ncols values
    and is refused without ncols, since its length alone does not tell 4 from 5 values per electron."""
    a = np.asarray(offsets, np.float64)
    if a.ndim == 2 and a.shape[1] in (4, 5) and ncols in (None, a.shape[1]):
        return np.ascontiguousarray(a)
    if a.ndim == 1 and ncols in (4, 5) and a.size % ncols == 0:
        return np.ascontiguousarray(a).reshape(-1, ncols)
    raise ValueError('electron offsets: an [n, 4] or [n, 5] array, or a flat array with ncols = 4 or 5 dividing its '
                     'length (got shape %s, ncols %s)' % (a.shape, ncols))


def _mesh_struct(m):
    """SRWLRadMesh from a dict or an object with the reference's mesh attribute names."""
    s = capi.SRWLRadMesh()
    get = (lambda k, d=None: m.get(k, d)) if isinstance(m, dict) else (lambda k, d=None: getattr(m, k, d))
    s.eStart = s.eFin = float(get('eStart', 0.))
    s.xStart, s.xFin, s.yStart, s.yFin = (float(get(k)) for k in ('xStart', 'xFin', 'yStart', 'yFin'))
    s.ne, s.nx, s.ny = 1, int(get('nx')), int(get('ny'))
    return s


class MultiE(object):
    def __init__(self, base_wfr, optC, acc_mesh, max_batch=8, graph=False, device=0):
        L = capi.lib()
        self._keep = []
        w = make_c_wfr(base_wfr, self._keep)
        self._optc = make_c_optc(optC, self._keep)      # must outlive the object (the library keeps it)
        self._accm = _mesh_struct(acc_mesh)
        h = C.c_void_p()
        capi.check(L.srwgMultiECreate(C.byref(w), C.byref(self._optc), C.byref(self._accm), int(max_batch),
                                      1 if graph else 0, int(device), C.byref(h)), 'multi-electron')
        self._h = h
        self.nx, self.ny = int(self._accm.nx), int(self._accm.ny)

    def add(self, offsets, stream=None, ncols=None):
        """offsets: [n, 4] (x, x', y, y') or [n, 5] with the relative energy deviation; a flat
        array needs ncols (4 or 5).  All electrons of a call are added, or none (on an error)."""
        off = offset_array(offsets, ncols)
        m = off.shape[1]
        st = C.c_void_p(stream) if stream else None
        f = capi.lib().srwgMultiEAddE if m == 5 else capi.lib().srwgMultiEAdd
        capi.check(f(self._h, int(off.shape[0]), off.ctypes.data, st), 'multi-electron add')

    def add_timed(self, offsets, stream=None, ncols=None):
        """Adds up to max_batch electrons as one batch without the graph and returns the device time
        [ms] of each pass and, last, of the accumulation (CUDA events on the stream)."""
        off = offset_array(offsets, ncols)
        ms = (C.c_float * 64)()
        n = C.c_int()
        st = C.c_void_p(stream) if stream else None
        capi.check(capi.lib().srwgMultiEAddTimed(self._h, int(off.shape[0]), off.ctypes.data, int(off.shape[1]), st,
                                                 ms, 64, C.byref(n)), 'multi-electron timed add')
        return [float(ms[i]) for i in range(min(n.value, 64))]

    def describe(self):
        """The planner's description of a batch's passes (the base electron's), as srwgPlanDescribe."""
        buf = C.create_string_buffer(1 << 16)
        capi.check(capi.lib().srwgMultiEInfo(self._h, None, None, buf, len(buf)), 'multi-electron info')
        return buf.value.decode()

    def info(self):
        """(passes of a batch [(kind, sizes...)] as Plan.kernels gives them, whether the last pass
        writes the intensity instead of the fields)."""
        from .plan import parse_passes
        n, i = C.c_int(), C.c_int()
        buf = C.create_string_buffer(1 << 16)
        capi.check(capi.lib().srwgMultiEInfo(self._h, C.byref(n), C.byref(i), buf, len(buf)), 'multi-electron info')
        ks = parse_passes(buf.value.decode())
        if len(ks) != n.value:
            raise RuntimeError('multi-electron info: %d passes described, %d planned' % (len(ks), n.value))
        return ks, bool(i.value)

    def count(self):
        n = C.c_longlong()
        capi.check(capi.lib().srwgMultiEGetMean(self._h, None, C.byref(n), None))
        return int(n.value)

    def mean(self, stream=None):
        out = np.empty((self.ny, self.nx), np.float64)
        n = C.c_longlong()
        st = C.c_void_p(stream) if stream else None
        capi.check(capi.lib().srwgMultiEGetMean(self._h, out.ctypes.data, C.byref(n), st), 'multi-electron mean')
        return out

    def accumulator(self):
        """(device address of the FP64 intensity sum [ny, nx], number of electrons added)."""
        p = C.c_void_p()
        n = C.c_longlong()
        capi.check(capi.lib().srwgMultiEAccumulator(self._h, C.byref(p), C.byref(n)))
        return int(p.value), int(n.value)

    def use_accumulator(self, dev_ptr):
        """Adds into caller-owned device memory (ny * nx float64, zeroed by the caller)."""
        capi.check(capi.lib().srwgMultiESetAccumulator(self._h, C.c_void_p(int(dev_ptr))))

    def reset(self):
        capi.check(capi.lib().srwgMultiEReset(self._h, None))

    def __del__(self):
        try:
            if getattr(self, '_h', None):
                capi.lib().srwgMultiEDestroy(self._h)
                self._h = None
        except Exception:
            pass
