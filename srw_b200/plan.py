"""Device-resident interface: plan a propagation once, run it on fields already in GPU memory.

    plan = Plan(wfr_template, optC)            # host bookkeeping, passes fixed
    out_x, out_y = plan.new_output()           # torch complex64 [ny_out, nx_out] on the GPU
    plan.execute(ex_in, ey_in, out_x, out_y)   # torch complex64 [ny_in, nx_in] inputs (read only)

Batches of wavefronts with the same mesh run back to back with ``execute_batch`` on tensors of
shape [B, ny, nx].  torch supplies device memory and streams only.
"""
import ctypes as C

import torch

from . import capi
from .srwlpy import make_c_optc, make_c_wfr


def parse_passes(text):
    """[(kind, sizes...), ...] of the passes in a plan description (srwgPlanDescribe's text):
    ('line_rows'|'line_cols', nx, ny), ('resize', nx_old, ny_old, nx_new, ny_new), ('moments', nx, ny)
    or ('pw', nx, ny)."""
    out = []
    for line in text.splitlines():
        f = line.split()
        if len(f) < 3:
            continue
        if f[1] == 'LINE':
            nx, ny = f[3].split('x')
            out.append(('line_' + f[2], int(nx), int(ny)))
        elif f[1] == 'RESIZE':
            nxo, nyo = f[2].split('x')
            nxn, nyn = f[4].split('x')
            out.append(('resize', int(nxo), int(nyo), int(nxn), int(nyn)))
        elif f[1] == 'MOM':
            nx, ny = f[2].split('x')
            out.append(('moments', int(nx), int(ny)))
        else:
            nx, ny = f[2].split('x')
            out.append(('pw', int(nx), int(ny)))
    return out


class Plan(object):
    def __init__(self, wfr, optC, device=0):
        L = capi.lib()
        keep = []
        w = make_c_wfr(wfr, keep)
        o = make_c_optc(optC, keep)
        h = C.c_void_p()
        capi.check(L.srwgPlanCreate(C.byref(w), C.byref(o), int(device), C.byref(h)), 'plan')
        self._h = h
        self.device = torch.device('cuda', int(device))
        a = [C.c_long() for _ in range(4)]
        nk = C.c_int()
        wb = C.c_longlong()
        capi.check(L.srwgPlanInfo(h, *[C.byref(x) for x in a], C.byref(nk), C.byref(wb)))
        self.nx_in, self.ny_in, self.nx_out, self.ny_out = [int(x.value) for x in a]
        self.n_kernels = int(nk.value)
        self.work_bytes = int(wb.value)
        self.out = capi.SRWLWfr()
        capi.check(L.srwgPlanGetOutput(h, C.byref(self.out)))

    def describe(self):
        buf = C.create_string_buffer(1 << 16)
        capi.lib().srwgPlanDescribe(self._h, buf, len(buf))
        return buf.value.decode()

    def output_mesh(self):
        m = self.out.mesh
        return dict(nx=int(m.nx), ny=int(m.ny), xStart=m.xStart, xFin=m.xFin, yStart=m.yStart, yFin=m.yFin,
                    Rx=self.out.Rx, Ry=self.out.Ry, dRx=self.out.dRx, dRy=self.out.dRy, xc=self.out.xc,
                    yc=self.out.yc, presCA=ord(self.out.presCA) if self.out.presCA else 0)

    def moments(self, index=0):
        """(momX, momY): the 11 + 11 output moments of wavefront `index` of the last execution (the
        analytically propagated ones when the plan recomputes none from the field)."""
        import numpy as np
        mx, my = np.zeros(11), np.zeros(11)
        capi.check(capi.lib().srwgPlanGetMoments(self._h, int(index), mx.ctypes.data, my.ctypes.data), 'moments')
        return mx, my

    def new_output(self, batch=None):
        shape = (self.ny_out, self.nx_out) if batch is None else (batch, self.ny_out, self.nx_out)
        return (torch.empty(shape, dtype=torch.complex64, device=self.device),
                torch.empty(shape, dtype=torch.complex64, device=self.device))

    def _check(self, t, shape):
        if t.dtype != torch.complex64 or not t.is_cuda or not t.is_contiguous() or tuple(t.shape[-2:]) != shape:
            raise ValueError('expected contiguous complex64 CUDA tensor of shape [..., %d, %d]' % shape)

    def execute(self, ex_in, ey_in, ex_out, ey_out, stream=None):
        for t in (ex_in, ey_in):
            self._check(t, (self.ny_in, self.nx_in))
        for t in (ex_out, ey_out):
            self._check(t, (self.ny_out, self.nx_out))
        st = (stream or torch.cuda.current_stream(self.device)).cuda_stream
        capi.check(capi.lib().srwgPlanExecute(self._h, ex_in.data_ptr(), ey_in.data_ptr(), ex_out.data_ptr(),
                                              ey_out.data_ptr(), C.c_void_p(st)), 'execute')

    def execute_timed(self, ex_in, ey_in, ex_out, ey_out, stream=None):
        """Runs once with a CUDA event pair around every pass; returns the per-pass times [ms]."""
        for t in (ex_in, ey_in):
            self._check(t, (self.ny_in, self.nx_in))
        for t in (ex_out, ey_out):
            self._check(t, (self.ny_out, self.nx_out))
        st = (stream or torch.cuda.current_stream(self.device)).cuda_stream
        ms = (C.c_float * max(1, self.n_kernels))()
        n = C.c_int()
        capi.check(capi.lib().srwgPlanExecuteTimed(self._h, ex_in.data_ptr(), ey_in.data_ptr(), ex_out.data_ptr(),
                                                   ey_out.data_ptr(), C.c_void_p(st), ms, len(ms), C.byref(n)),
                   'execute_timed')
        return [float(ms[i]) for i in range(n.value)]

    def kernels(self):
        """[(kind, nx, ny), ...] of the planned passes, parsed from describe()."""
        return parse_passes(self.describe())

    def execute_batch(self, ex_in, ey_in, ex_out, ey_out, stream=None):
        B = ex_in.shape[0]
        for t in (ex_in, ey_in):
            self._check(t, (self.ny_in, self.nx_in))
        for t in (ex_out, ey_out):
            self._check(t, (self.ny_out, self.nx_out))
        st = (stream or torch.cuda.current_stream(self.device)).cuda_stream
        si = 2 * self.nx_in * self.ny_in
        so = 2 * self.nx_out * self.ny_out
        capi.check(capi.lib().srwgPlanExecuteBatch(self._h, int(B), ex_in.data_ptr(), ey_in.data_ptr(), si,
                                                   ex_out.data_ptr(), ey_out.data_ptr(), so, C.c_void_p(st)),
                   'execute_batch')

    def __del__(self):
        try:
            if getattr(self, '_h', None):
                capi.lib().srwgPlanDestroy(self._h)
                self._h = None
        except Exception:
            pass
