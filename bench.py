"""Benchmark: propagation of the 1024^2 undulator beamline on B200, batched and single-wavefront.

Workload (the configuration the headline metric is quoted on): a 1024x1024 complex-FP32
undulator-like wavefront (first harmonic of a 3 GeV, K=1.5, 100 x 20 mm planar undulator seen at
20 m, 2012 eV, +-1.5 mm; synthetic, see synth_undulator_field) through a 0.8 mm circular aperture,
a thin lens f=10 m with range x2 / resolution x2 resizing before it (-> 4096^2), and a 10 m drift
to the waist (to-waist mode).

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Prints one JSON line.  ``value`` is propagations/s of the batched path with learned resize factors:
one step = a batch of BATCH macro-electron wavefronts (the field with each electron's source offset,
made on the device) propagated together and their intensities added in FP64 on the device, with the
range / resolution factors the trained network (srw_b200.learned) chooses -- when its choice passes
the run-time check and the mean intensity agrees within 1e-3 with the configured factors' (2, 2) on
the same electrons; otherwise the configured factors (``batched_configured``).  ``plain`` is the
single-wavefront path (one propagation per step, device-resident field) with the per-pass CUDA
event times that give ``roofline``.  ``e2e`` is the batched path through its public API (electron
offsets from the host in, mean intensity to the host out, every step); ``e2e_single_wavefront`` is
the srwlpy-compatible C-ABI call with pinned host buffers.  ``mixed_grid_multi_electron`` runs
electrons on 256^2 / 512^2 / 1024^2 grids batched and one at a time.  ``--impl reference`` times
the reference SRW (built from source, FFTW3 CPU path) on the host cores.
"""
import argparse
import json
from array import array
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "propagations/s at 1024² FP32, batched+learned vs plain GPU at ≤1e-3 rel err"
UNIT = "propagations/s"
WORKLOAD = ("undulator beamline: 1024x1024 complex FP32 field (2012 eV, +-1.5 mm, R=20 m) -> circular aperture "
            "0.8 mm -> resize x2 range x2 resolution (4096x4096) -> thin lens f=10 m -> drift 10 m to waist; "
            "macro-electron wavefronts (source offsets sigma x 30 um, x' 5 urad, y 5 um, y' 2 urad; relative energy "
            "spread 1e-3 as a photon-energy rescale E (1 + 2 d)) in batches")
PEAKS = os.path.join(HERE, 'MEASURED_PEAKS.json')
BATCH = 16                                     # macro-electron wavefronts per step
SIG = (30e-6, 5e-6, 5e-6, 2e-6)                # source: sigma x [m], x' [rad], y [m], y' [rad]
SIG_E = 1e-3                                   # relative electron energy spread (photon energy E (1 + 2 d))
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one launch of a pass, from an ncu
# capture of this workload (the plain passes' summary under profiles/); keyed by the pass tuple of
# Plan.kernels().  Re-captured whenever the kernel changes.
TRAFFIC = {('line_cols', 4096, 4096): 37369856 + 216899840,
           ('line_rows', 4096, 4096): 5258752 + 2144256,
           ('resize', 1024, 1024, 4096, 4096): 1373696 + 512}
# the same per electron of the batched passes at the learned factors (ncu on a batch of 8, the
# learned batch's summary under profiles/); a launch moves this times its electrons
TRAFFIC_PER_ELECTRON = {('line_cols', 1536, 1600): (69851904 + 29201664) // 8,
                        ('line_rows', 1536, 1600): (19814912 + 20619776) // 8,
                        ('resize', 1024, 1024, 1536, 1600): (2238208 + 202240) // 8}


# ------------------------------------------------------------------------------------------------
# synthetic input (same for both arms)
# ------------------------------------------------------------------------------------------------
def synth_undulator_field(n=1024, r=1.5e-3, z=20.):
    """Undulator-like first-harmonic field at distance z: on-resonance detuning ring structure
    sinc(q) exp(-i pi q), q = N gamma^2 theta^2 / (1 + K^2/2), on a spherical wave of radius z,
    plus a weak vertical component.  Deterministic (no RNG)."""
    per, nper, K = 0.02, 100, 1.5
    gam = 3. / 0.51099890221e-03
    lam1 = per / (2. * gam * gam) * (1. + K * K / 2.)
    E = 1.239842e-06 / lam1
    x = np.linspace(-r, r, n)
    X, Y = np.meshgrid(x, x)
    th2 = (X * X + Y * Y) / (z * z)
    q = nper * gam * gam * th2 / (1. + K * K / 2.)
    amp = 3.0e7 * np.sinc(q) * np.exp(-1j * np.pi * q)
    sph = np.exp(1j * np.pi * (X * X + Y * Y) / (lam1 * z))
    ex = (amp * sph).astype(np.complex64)
    ey = (0.02 * amp * sph * (X * Y) / (r * r)).astype(np.complex64)
    mesh = dict(nx=n, ny=n, xStart=-r, xFin=r, yStart=-r, yFin=r, eStart=E, eFin=E, zStart=z)
    return ex, ey, mesh, dict(Rx=z, Ry=z, dRx=0.01 * z, dRy=0.01 * z)


CONFIGURED = (2., 2., 2., 2.)     # pxm, pxd, pzm, pzd of the resize before the lens, as configured


def beamline_objs(mod, fac=CONFIGURED):
    """C1 beamline with classes from module `mod` (srw_b200.srwlib, or the reference's when given);
    fac = range / resolution factors (pxm, pxd, pzm, pzd) of the resize before the lens."""
    pp = lambda anal=0, f=(1., 1., 1., 1.): [0, 0, 1., anal, 0, f[0], f[1], f[2], f[3], 0, 0, 0]  # noqa: E731
    return mod.SRWLOptC([mod.SRWLOptA('c', 'a', 0.8e-3, 0.8e-3), mod.SRWLOptL(10., 10.), mod.SRWLOptD(10.)],
                        [pp(), pp(0, tuple(fac)), pp(4)])


def make_wfr(mod, ex, ey, mesh, sc, alloc=None):
    w = mod.SRWLWfr()
    w.allocate(1, mesh['nx'], mesh['ny'])
    for name, f in (('arEx', ex), ('arEy', ey)):
        a = np.empty(2 * f.size, np.float32) if alloc is None else alloc(2 * f.size)
        a[0::2] = f.real.ravel()
        a[1::2] = f.imag.ravel()
        setattr(w, name, a)
    for k in ('xStart', 'xFin', 'yStart', 'yFin', 'eStart', 'eFin', 'zStart'):
        setattr(w.mesh, k, mesh[k])
    w.Rx, w.Ry, w.dRx, w.dRy = sc['Rx'], sc['Ry'], sc['dRx'], sc['dRy']
    return w


# ------------------------------------------------------------------------------------------------
# clocks sampled during the timed region
# ------------------------------------------------------------------------------------------------
class NvmlSampler(object):
    """Polls SM clock, max clock and clock-event reasons through NVML every `period` seconds
    (read-only queries) while the timed region runs."""
    REASONS = {0x8: 'hw_slowdown', 0x40: 'hw_thermal_slowdown', 0x20: 'sw_thermal_slowdown',
               0x4: 'sw_power_cap', 0x80: 'hw_power_brake_slowdown'}

    def __init__(self, torch_dev, period=0.01):
        self.dev, self.period, self.rows, self.h = torch_dev, period, [], None
        self.stop = threading.Event()

    def __enter__(self):
        try:
            import pynvml as N
            import torch
            N.nvmlInit()
            self.N = N
            p = torch.cuda.get_device_properties(self.dev)
            try:
                bus = '%08X:%02X:%02X.0' % (p.pci_domain_id, p.pci_bus_id, p.pci_device_id)
                self.h = N.nvmlDeviceGetHandleByPciBusId(bus)
            except Exception:
                self.h = N.nvmlDeviceGetHandleByIndex(self.dev.index)
            self.mx = float(N.nvmlDeviceGetMaxClockInfo(self.h, N.NVML_CLOCK_SM))
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
        except Exception:
            self.h = None
        return self

    def _poll(self):
        N = self.N
        while not self.stop.is_set():
            try:
                sm = float(N.nvmlDeviceGetClockInfo(self.h, N.NVML_CLOCK_SM))
                rs = int(N.nvmlDeviceGetCurrentClocksEventReasons(self.h))
                self.rows.append((sm, rs))
            except Exception:
                pass
            time.sleep(self.period)

    def __exit__(self, *a):
        self.stop.set()
        if self.h is not None:
            self.t.join(timeout=2)

    def summary(self):
        if not self.rows:
            return None
        reasons = sorted({n for _, r in self.rows for b, n in self.REASONS.items() if r & b})
        return {"sm_mhz": statistics.median([r[0] for r in self.rows]), "sm_max_mhz": self.mx, "reasons": reasons,
                "samples": len(self.rows), "source": "nvml, 10 ms period"}


class ClockSampler(object):
    Q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,'
         'clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,'
         'clocks_event_reasons.sw_power_cap')

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.idx), '--query-gpu=' + self.Q,
                                          '--format=csv,noheader,nounits', '-lms', '200'],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(',')])

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace('.', '', 1).isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace('.', '', 1).isdigit()]
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        reasons = sorted({names[k] for r in self.rows if len(r) > 8 for k in range(4) if r[5 + k] == 'Active'})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ------------------------------------------------------------------------------------------------
# reference arm: the reference SRW built from source (oracle/_ref/srwlpy.so), CPU
# ------------------------------------------------------------------------------------------------
REF_PROC_BYTES = 600 << 20       # host memory of one reference propagation of this workload (max RSS 351 MB)


def _ref_worker(args):
    """One propagation with the reference's own srwlpy (runs in a spawned process); `ref_dir` is the
    MODE=0 build (oracle/_ref) or the OpenMP build (oracle/_ref/omp)."""
    ref_dir, n = args
    sys.path.insert(0, ref_dir)
    import srwlpy
    from srw_b200 import srwlib as mod          # plain Python structures with the reference's names
    ex, ey, mesh, sc = synth_undulator_field(n)
    w = make_wfr(mod, ex, ey, mesh, sc)
    t = time.perf_counter()
    srwlpy.PropagElecField(w, beamline_objs(mod))
    return time.perf_counter() - t, int(w.mesh.nx)


def reference_available(omp=False):
    d = os.path.join(HERE, 'oracle', '_ref', 'omp' if omp else '')
    d = os.path.normpath(d)
    return d if os.path.exists(os.path.join(d, 'srwlpy.so')) else None


def host_info():
    """Host cores, CPU model, OpenMP setting and available memory (the reference arm's context)."""
    model = None
    try:
        out = subprocess.run(['lscpu'], capture_output=True, text=True, timeout=10).stdout
        model = next((l.split(':', 1)[1].strip() for l in out.splitlines() if l.startswith('Model name')), None)
    except Exception:
        pass
    if model is None and os.path.exists('/proc/cpuinfo'):
        model = next((l.split(':', 1)[1].strip() for l in open('/proc/cpuinfo') if l.startswith('model name')), None)
    avail = None
    try:
        import psutil
        avail = psutil.virtual_memory().available
    except Exception:
        pass
    return {"nproc": os.cpu_count(), "cpu_model": model, "OMP_NUM_THREADS": os.environ.get('OMP_NUM_THREADS'),
            "mem_available_bytes": avail}


def reference_procs():
    """Processes for the reference arm: every host core, capped by available memory at
    REF_PROC_BYTES per propagation."""
    info = host_info()
    procs = info['nproc'] or 1
    cap = None
    if info['mem_available_bytes']:
        cap = max(1, int(info['mem_available_bytes'] // REF_PROC_BYTES))
        procs = min(procs, cap)
    return procs, cap, info


def _time_pool(ref, procs, n, omp_threads=None):
    """Per-propagation times of n propagations in a pool of `procs` spawned processes."""
    import multiprocessing as mp
    env_old = os.environ.get('OMP_NUM_THREADS')
    if omp_threads:
        os.environ['OMP_NUM_THREADS'] = str(omp_threads)
    try:
        with mp.get_context('spawn').Pool(procs) as pool:
            return [r[0] for r in pool.map(_ref_worker, [(ref, 1024)] * n)]
    finally:
        if omp_threads:
            if env_old is None:
                os.environ.pop('OMP_NUM_THREADS', None)
            else:
                os.environ['OMP_NUM_THREADS'] = env_old


def cpu_baseline_sample(n_props=5):
    """Times the reference CPU path (MODE=0 build: FFTW3, one thread) on the same workload: n_props
    propagations, each in its own single-threaded process (run side by side); the value is one core's
    propagations/s from the median time."""
    ref = reference_available()
    if ref is None:
        return None
    ts = _time_pool(ref, n_props, n_props)
    med = statistics.median(ts)
    return {"value": 1. / med, "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": "%d full propagations of the same 1024^2 workload with the reference SRW (MODE=0 build from "
                      "source: FFTW 3.3.8, single-threaded), one per process side by side; median %.2f s per "
                      "propagation (min %.2f, max %.2f)" % (n_props, med, min(ts), max(ts)),
            "host": host_info()}


def run_reference(args, rank, world):
    if rank != 0:
        return
    ref = reference_available()
    if ref is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref/srwlpy.so not present"}))
        return
    import multiprocessing as mp
    procs, cap, info = reference_procs()
    ctx = mp.get_context('spawn')
    times, per = [], []
    with ctx.Pool(procs) as pool:
        for i in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            res = pool.map(_ref_worker, [(ref, 1024)] * procs)
            dt = time.perf_counter() - t0
            if i >= args.warmup:
                times.append(dt)
                per += [r[0] for r in res]
    total = sum(times)
    value = procs * len(times) / total
    # the reference's OpenMP build (FFTW 2.1.5 + OpenMP loops, cpp/gcc/Makefile:43-45), one process
    # with a thread per core: a few propagations, reported beside the arm's value
    omp = None
    ref_omp = reference_available(omp=True)
    if ref_omp is not None:
        nth = info['nproc'] or 1
        ts = _time_pool(ref_omp, 1, 3, omp_threads=nth)
        omp = {"value": 1. / statistics.median(ts[1:]), "unit": UNIT, "OMP_NUM_THREADS": nth,
               "sample": "3 propagations in one process (first one a warm-up), median of the last two",
               "seconds": ts}
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1000. * total / len(times), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
           "config": {"workload": WORKLOAD, "step": "%d concurrent reference propagations (one per process, MODE=0 "
                                                    "build: FFTW 3.3.8, single-threaded)" % procs},
           "impl": "reference",
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": "reference",
                            "sample": "each step: %d processes x 1 propagation of the full workload (all %s host "
                                      "cores%s); median %.2f s per propagation" % (
                                          procs, info['nproc'],
                                          ", capped at %d by available memory" % cap if cap and cap < (info['nproc'] or 1)
                                          else "", statistics.median(per))},
           "host": info, "omp_build": omp,
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


# ------------------------------------------------------------------------------------------------
# our arm
# ------------------------------------------------------------------------------------------------
def kernel_bytes(k):
    """Algorithmic bytes of one pass (both components, read + write, complex FP32)."""
    if k[0] == 'resize':
        return 2 * 8 * (k[1] * k[2] + k[3] * k[4])
    return 2 * 8 * 2 * k[1] * k[2]


def hbm_peak():
    """(HBM GB/s, 'measured' | 'fallback'): the measured copy bandwidth of this GPU pool when the
    peaks file is present, else the earlier measured fallback figure."""
    if os.path.exists(PEAKS):
        return float(json.load(open(PEAKS))['hbm_gbs']), 'measured'
    return 6650., 'fallback'


def batched_passes(me, offs, stream, peak, peak_src, where):
    """One batch of the multi-electron object `me` (MultiE) run without its graph, with CUDA events
    around every pass (srwgMultiEAddTimed; adds the electrons): per-pass times and the roofline of the
    dominant pass -- algorithmic bytes per electron (kernel_bytes; a last pass that writes the
    intensity writes one float per point instead of two complex values) times the electrons of the
    launch, over the pass's CUDA-event time."""
    ks, inten = me.info()
    ms = me.add_timed(offs, stream)
    nb = len(offs)
    per = ms[:len(ks)]
    alg = [kernel_bytes(k) for k in ks]
    if inten:
        k = ks[-1]
        alg[-1] = 2 * 8 * k[1] * k[2] + 4 * k[1] * k[2]
    kd = int(np.argmax(per))
    achieved = alg[kd] * nb / (per[kd] / 1000.) / 1e9
    return {"bound": "hbm", "kernel": "%s %s (batch of %d)" % (ks[kd][0], 'x'.join(map(str, ks[kd][1:])), nb),
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_src,
            "traffic": (TRAFFIC_PER_ELECTRON[tuple(ks[kd])] * nb if tuple(ks[kd]) in TRAFFIC_PER_ELECTRON else None),
            "algorithmic_bytes": alg[kd] * nb, "avg_ms": float(per[kd]),
            "per_pass_ms": [round(float(v), 4) for v in per], "accumulation_ms": round(float(ms[-1]), 4),
            "per_electron_ms": round(float(sum(ms)) / nb, 5), "passes": [list(k) for k in ks],
            "last_pass_writes_intensity": inten, "measured_on": where}


def measure_plain(args, dev, world, dist, factors=CONFIGURED):
    """Single-wavefront path: one propagation per step on a device-resident field, CUDA events per
    step and per pass (roofline), L2 flushed between steps; `factors`: the resize before the lens."""
    import torch
    from srw_b200 import srwlib as mod
    from srw_b200.plan import Plan
    ex, ey, mesh, sc = synth_undulator_field(1024)
    w = make_wfr(mod, ex, ey, mesh, sc)
    plan = Plan(w, beamline_objs(mod, factors), device=dev.index)
    dex = torch.from_numpy(ex).to(dev)
    dey = torch.from_numpy(ey).to(dev)
    ox, oy = plan.new_output()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)    # > L2 (126 MB)
    stream = torch.cuda.current_stream(dev)
    kinfo = plan.kernels()
    for _ in range(args.warmup):
        plan.execute(dex, dey, ox, oy)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    steps = max(3, args.steps // 2)
    step_ms, kern_ms = [], []
    for _ in range(steps):
        flush.fill_(1)                                      # L2 flush between steps (outside the events)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        kern_ms.append(plan.execute_timed(dex, dey, ox, oy, stream))
        e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
    torch.cuda.synchronize(dev)
    total_ms = _max_over_ranks(sum(step_ms), dev, world, dist)
    per_k = np.mean(np.array(kern_ms), axis=0)
    return dict(plan=plan, kinfo=kinfo, per_k=per_k, steps=steps, total_ms=total_ms,
                value=world * steps / (total_ms / 1000.))


def measure_with_input_moments(args, dev):
    """The plain path on the same field carrying statistical moments, as a source calculation leaves
    them (norm, centre and rms sizes of the intensity; zero angular moments): the aperture's 1.7 sigma
    check then fails and the moment pass recomputes them from the field.  Per-pass CUDA events."""
    import torch
    from srw_b200 import srwlib as mod
    from srw_b200.plan import Plan
    ex, ey, mesh, sc = synth_undulator_field(1024)
    I = np.abs(ex.astype(np.complex128)) ** 2 + np.abs(ey.astype(np.complex128)) ** 2
    x = np.linspace(mesh['xStart'], mesh['xFin'], mesh['nx'])[None, :]
    y = np.linspace(mesh['yStart'], mesh['yFin'], mesh['ny'])[:, None]
    n = I.sum()
    xm, ym = float((I * x).sum() / n), float((I * y).sum() / n)
    mom = [float(n), xm, 0., ym, 0., float((I * x * x).sum() / n), 0., 0., float((I * y * y).sum() / n), 0., 0.]
    w = make_wfr(mod, ex, ey, mesh, sc)
    w.arMomX = array('d', mom)
    w.arMomY = array('d', mom)
    plan = Plan(w, beamline_objs(mod), device=dev.index)
    dex = torch.from_numpy(ex).to(dev)
    dey = torch.from_numpy(ey).to(dev)
    ox, oy = plan.new_output()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        plan.execute(dex, dey, ox, oy)
    ms = []
    for _ in range(max(3, args.steps // 4)):
        flush.fill_(1)
        ms.append(plan.execute_timed(dex, dey, ox, oy, stream))
    torch.cuda.synchronize(dev)
    per = np.mean(np.array(ms), axis=0)
    kinds = [k[0] for k in plan.kernels()]
    return {"passes": kinds, "per_pass_ms": [round(float(v), 4) for v in per],
            "ms_per_propagation": round(float(per.sum()), 4),
            "moment_pass_ms": round(float(sum(v for k, v in zip(kinds, per) if k == 'moments')), 4),
            "path": "srwgPlanExecute, input with moments: the aperture recomputes them on the device"}


def _max_over_ranks(v, dev, world, dist):
    if world <= 1:
        return v
    import torch
    t = torch.tensor([v], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _acc_mesh(plan, n=512):
    om = plan.output_mesh()
    return dict(nx=n, ny=n, xStart=om['xStart'], xFin=om['xFin'], yStart=om['yStart'], yFin=om['yFin'])


def measure_batched(args, dev, world, dist, factors=CONFIGURED, acc=None, e2e_leg=True):
    """Batched path: each step propagates a batch of BATCH macro-electron wavefronts (the 1024^2
    field offset per electron) through the same beamline and adds their intensities on the device;
    K steps between two CUDA events (host planning of the electrons included)."""
    import torch
    from srw_b200 import srwlib as mod
    from srw_b200.multie import MultiE, sample_offsets
    from srw_b200.plan import Plan
    ex, ey, mesh, sc = synth_undulator_field(1024)
    w = make_wfr(mod, ex, ey, mesh, sc)
    bl = beamline_objs(mod, factors)
    acc = acc or _acc_mesh(Plan(w, beamline_objs(mod), device=dev.index))
    me = MultiE(w, bl, acc, max_batch=BATCH, graph=True, device=dev.index)
    # the FP64 intensity sum lives in a torch tensor so that ranks can sum it (NCCL) at the end
    acc_t = torch.zeros((acc['ny'], acc['nx']), dtype=torch.float64, device=dev)
    me.use_accumulator(acc_t.data_ptr())
    # a stream of its own: batches are queued without host synchronisation (the legacy default
    # stream cannot be captured into a graph)
    stream = torch.cuda.Stream(dev)
    torch.cuda.synchronize(dev)
    rank = int(os.environ.get('RANK', '0'))
    for k in range(args.warmup):
        me.add(sample_offsets(BATCH, *SIG, seed=1000 + rank, first=k * BATCH, sig_e=SIG_E), stream.cuda_stream)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    offs = [sample_offsets(BATCH, *SIG, seed=rank, first=k * BATCH, sig_e=SIG_E) for k in range(args.steps)]
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index) as clk, NvmlSampler(dev) as nv:
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for k in range(args.steps):
            me.add(offs[k], stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize(dev)
    total_ms = _max_over_ranks(e0.elapsed_time(e1), dev, world, dist)
    value = world * args.steps * BATCH / (total_ms / 1000.)
    if world > 1:
        dist.all_reduce(acc_t)                   # mean intensity over all ranks' electrons
    n_all = world * (args.warmup + args.steps) * BATCH
    mean_peak = float(acc_t.max().item()) / n_all
    mean = acc_t.cpu().numpy() / n_all
    peak, peak_src = hbm_peak()
    passes = batched_passes(me, offs[0], stream.cuda_stream, peak, peak_src,
                            "batched leg (configured factors), one batch of %d electrons, CUDA events per pass" % BATCH)

    # end to end through the public API: host offsets in, mean intensity (host) out, every step
    e2e = None
    if e2e_leg and not args.no_e2e:
        me2 = MultiE(w, bl, acc, max_batch=BATCH, graph=True, device=dev.index)
        me2.add(sample_offsets(BATCH, *SIG, seed=77, sig_e=SIG_E))
        me2.mean()
        n_e2e = max(3, min(args.steps, 20))
        t0 = time.perf_counter()
        for k in range(n_e2e):
            me2.add(offs[k % len(offs)])
            mean = me2.mean()
        e2e_s = time.perf_counter() - t0
        e2e = {"value": world * n_e2e * BATCH / e2e_s, "unit": UNIT, "h2d_bytes_per_step": BATCH * 5 * 8,
               "d2h_bytes_per_step": int(mean.nbytes),
               "path": "srw_b200.multie.MultiE.add (C-ABI srwgMultiEAdd; base field resident, electron offsets "
                       "from host) + MultiE.mean (D2H of the %dx%d FP64 mean intensity)" % (acc['nx'], acc['ny'])}
    return dict(value=value, total_ms=total_ms, e2e=e2e, clocks=nv.summary() or clk.summary(), mean_peak=mean_peak,
                n_all=n_all, mean=mean, acc=acc, passes=passes)


def measure_mixed(args, dev, n_elec, model=None):
    """Partially coherent workload: n_elec electrons, grids 256^2 / 512^2 / 1024^2 in equal numbers,
    batched (one MultiE per grid class, graphs) against the same electrons one at a time, and
    batched with the factors the trained network chooses per grid class (mean intensity compared
    with the configured factors' on the same electrons)."""
    import torch
    from srw_b200 import srwlib as mod
    from srw_b200.multie import MultiE, sample_offsets
    from srw_b200.plan import Plan
    modes = [('batched', None, True), ('plain', 1, False)]
    if model is not None:
        modes.append(('learned', None, True))
    res, errs, facs = {}, {}, {}
    means = {}
    for mode, batch, graph in modes:
        total = 0.
        for cls, n in enumerate((256, 512, 1024)):
            ex, ey, mesh, sc = synth_undulator_field(n)
            w = make_wfr(mod, ex, ey, mesh, sc)
            acc = _acc_mesh(Plan(w, beamline_objs(mod), device=dev.index))
            factors = CONFIGURED
            if mode == 'learned':
                from srw_b200 import learned
                chk_set = sample_offsets(N_CHECK, *SIG, seed=31337 + n, sig_e=SIG_E)
                factors, fb, _ = learned.choose_factors(model, learned.bench_case(ex, ey, mesh, sc), dev,
                                                        acc_mesh=acc, check_offsets=chk_set, refine=REFINE)
                facs[n] = list(factors) + (['fallback'] if fb else [])
            bl = beamline_objs(mod, factors)
            b = batch or {256: 32, 512: 32, 1024: 16}[n]
            if mode == 'learned':
                # the mean intensity of the check set (grown by one electron per batch) checked before every batch
                me = learned.CheckedMultiE(w, lambda f: beamline_objs(mod, f), factors, acc,
                                           max_batch=LEARNED_BATCH, launch_batch=LEARNED_LAUNCH, graph=graph,
                                           device=dev.index, check_offsets=chk_set)
                me.add(sample_offsets(LEARNED_LAUNCH, *SIG, seed=999, sig_e=SIG_E))     # warm-up (plans, graph)
                me.reset()
            else:
                me = MultiE(w, bl, acc, max_batch=b, graph=graph, device=dev.index)
                me.add(sample_offsets(b, *SIG, seed=999, sig_e=SIG_E))                  # warm-up (plans, graph)
                me.reset()
            cnt = n_elec // 3
            offs = sample_offsets(cnt, *SIG, seed=5, first=cls * cnt, sig_e=SIG_E)
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            me.add(offs)
            if mode == 'learned':
                me.resolve()
            torch.cuda.synchronize(dev)
            total += time.perf_counter() - t0
            m = me.mean()
            if mode == 'batched':
                means[n] = m
            elif mode == 'learned':
                ref = means[n]
                sel = ref > 1e-3 * ref.max()
                errs[n] = float(np.linalg.norm(m[sel] - ref[sel]) / np.linalg.norm(ref[sel]))
        res[mode] = 3 * (n_elec // 3) / total
    out = {"electrons": 3 * (n_elec // 3), "grids": [256, 512, 1024], "unit": "electrons/s",
           "batched": res['batched'], "plain": res['plain'], "speedup": res['batched'] / res['plain'],
           "note": "each electron: offset field, C1 beamline (resize before the lens), intensity added in FP64 "
                   "onto a 512x512 common mesh; plain = the same electrons one per launch sequence with the "
                   "configured factors (2, 2); learned = per grid class the network's factors (checked on the mean "
                   "intensity of a 32-electron check set), checked batches of 256 launched 64 at a time, the first "
                   "electron of every batch added to the check set at both factors and the check repeated"}
    if model is not None:
        out.update({"batched_learned": res['learned'], "learned_speedup_vs_plain": res['learned'] / res['plain'],
                    "learned_factors": {str(k): v for k, v in facs.items()},
                    "learned_rel_err_vs_configured": {str(k): v for k, v in errs.items()}})
    return out


LEARNED_BATCH = 256              # macro-electron wavefronts per step of the learned leg (one checked batch)
LEARNED_LAUNCH = 64              # electrons per launch inside it (the device starts while the host plans the rest)
N_CHECK = 32                     # electrons of the learned factors' check set
REFINE = 4                       # checks spent lowering the resolution of a passing choice


def load_model(dev):
    """The packaged resize-factor network, or None when it is missing or was trained for other features."""
    from srw_b200 import learned
    if not os.path.exists(learned.DEFAULT_MODEL):
        return None
    m = learned.ResizeMLP.load(learned.DEFAULT_MODEL, device=dev.index)
    return m if (m.sizes[0] == learned.N_IN and m.sizes[-1] == learned.N_OUT) else None


def measure_learned(args, dev, world, dist, acc):
    """Batched path with the resize factors the trained network chooses for this wavefront and
    beamline (srw_b200.learned.choose_factors: the mean intensity of a seeded check set of N_CHECK
    electrons propagated with them checked against the conservative factors', fallback above 1e-3),
    run through learned.CheckedMultiE: batches of LEARNED_BATCH electrons (launched LEARNED_LAUNCH at a
    time), the first electron of every batch added to the check set at both factors and the check repeated before the batch (above 1e-3
    the run falls back to the conservative factors for good).  K steps between CUDA events, checks
    included."""
    import torch
    from srw_b200 import learned
    from srw_b200 import srwlib as mod
    from srw_b200.multie import sample_offsets
    model = load_model(dev)
    if model is None:
        return None
    ex, ey, mesh, sc = synth_undulator_field(1024)
    chk_set = sample_offsets(N_CHECK, *SIG, seed=31337, sig_e=SIG_E)
    trace = []
    t0 = time.perf_counter()
    factors, fallback, chk = learned.choose_factors(model, learned.bench_case(ex, ey, mesh, sc), dev, acc_mesh=acc,
                                                    check_offsets=chk_set, trace=trace, refine=REFINE)
    choose_s = time.perf_counter() - t0
    w = make_wfr(mod, ex, ey, mesh, sc)
    cm = learned.CheckedMultiE(w, lambda f: beamline_objs(mod, f), factors, acc, max_batch=LEARNED_BATCH,
                               graph=True, device=dev.index, check_offsets=chk_set, launch_batch=LEARNED_LAUNCH)
    stream = torch.cuda.Stream(dev)
    rank = int(os.environ.get('RANK', '0'))
    for k in range(args.warmup):
        cm.add(sample_offsets(LEARNED_BATCH, *SIG, seed=2000 + rank, first=k * LEARNED_BATCH, sig_e=SIG_E),
               stream.cuda_stream)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    offs = [sample_offsets(LEARNED_BATCH, *SIG, seed=rank, first=k * LEARNED_BATCH, sig_e=SIG_E)
            for k in range(args.steps)]
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with NvmlSampler(dev) as nv:
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for k in range(args.steps):
            cm.add(offs[k], stream.cuda_stream)
        cm.resolve(stream.cuda_stream)              # the last checks (a failure reruns inside the timing)
        e1.record(stream)
        torch.cuda.synchronize(dev)
    total_ms = _max_over_ranks(e0.elapsed_time(e1), dev, world, dist)
    value = world * args.steps * LEARNED_BATCH / (total_ms / 1000.)
    ce = list(cm.check_errors)
    fell_back, rerun, n_check = cm.fell_back, cm.rerun, cm.n_check
    # end to end through the public API: host offsets in, the mean intensity (host) out, every step
    e2e = None
    if not args.no_e2e:
        for k in range(max(1, args.warmup)):     # untimed: the object's own stream and its buffers
            cm.add(sample_offsets(LEARNED_BATCH, *SIG, seed=3000 + rank, first=k * LEARNED_BATCH, sig_e=SIG_E))
            cm.mean()
        n_e2e = max(3, min(args.steps, 20))
        t0 = time.perf_counter()
        for k in range(n_e2e):
            cm.add(offs[k % len(offs)])
            mean = cm.mean()
        e2e_s = time.perf_counter() - t0
        e2e = {"value": world * n_e2e * LEARNED_BATCH / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": int(offs[0].nbytes), "d2h_bytes_per_step": int(mean.nbytes),
               "path": "srw_b200.learned.CheckedMultiE.add (C-ABI srwgMultiEAdd; base field resident, electron "
                       "offsets from host, the run-time check included) + CheckedMultiE.mean (D2H of the %dx%d FP64 "
                       "mean intensity)" % (acc['nx'], acc['ny'])}
    peak, peak_src = hbm_peak()
    passes = batched_passes(cm.safe if cm.fell_back else cm.fast, offs[0][:LEARNED_LAUNCH], stream.cuda_stream, peak,
                            peak_src, "learned leg, one launch of %d electrons, CUDA events per pass" % LEARNED_LAUNCH)
    from srw_b200.plan import Plan
    nk_f = Plan(w, beamline_objs(mod, factors), device=dev.index).n_kernels
    nk_c = Plan(w, beamline_objs(mod), device=dev.index).n_kernels
    return {"value": value, "unit": UNIT, "ms_per_step": total_ms / args.steps, "batch": LEARNED_BATCH,
            # per step: the batch's launches and the checked electron (kick, passes, accumulation each),
            # and the checked electron with the conservative factors
            "launches_per_step": (LEARNED_BATCH // LEARNED_LAUNCH + 1) * (nk_f + 2) + (nk_c + 2),
            "launch_batch": LEARNED_LAUNCH,
            "factors": list(factors), "configured_factors": list(CONFIGURED),
            "fallback": bool(fallback or fell_back),
            "choice_check_rel_err": chk, "choose_seconds": choose_s,
            "choice_trace": [[list(f), e] for f, e in trace],
            "choice_check": "mean intensity of %d electrons (seeded check set) on the detector mesh, candidate vs "
                            "conservative factors, relative L2 where the conservative one exceeds 1e-3 of its "
                            "maximum; tolerance %g" % (N_CHECK, learned.TOL_LABEL),
            "run_checks": {"batches": len(ce), "fell_back": bool(fell_back), "rerun_electrons": rerun,
                           "check_electrons": n_check, "max_rel_err": max(ce) if ce else None,
                           "last_rel_err": ce[-1] if ce else None,
                           "what": "with every batch, queued behind it: the check set (the choice's electrons plus "
                                   "the first electron of every batch so far) at both factors, relative L2 of the two "
                                   "mean intensities, read when the batch after next is queued; above the tolerance "
                                   "the run falls back to the conservative factors for good and propagates the "
                                   "learned batches again"},
            "clocks": nv.summary(), "passes": passes, "e2e": e2e,
            "model": {k: v for k, v in getattr(model, 'meta', {}).items()
                      if k in ('samples', 'val_grid_at_least_label', 'val_cost_pred', 'labels_conservative', 'tol')}}


# ------------------------------------------------------------------------------------------------
# error of the batched (and learned) mean intensity against the FP64 oracle (outside the timed region)
# ------------------------------------------------------------------------------------------------
N_ORACLE = 16                    # electrons of the oracle comparison
ORACLE_PROC_BYTES = 5 << 30      # host memory of one oracle propagation of this workload (max RSS 4.3 GB)


def oracle_beamline(fac=CONFIGURED):
    """The beamline of beamline_objs as the oracle's element tuples and propagation parameters."""
    pp = lambda anal=0, f=(1., 1., 1., 1.): [0, 0, 1., anal, 0, f[0], f[1], f[2], f[3], 0, 0, 0]  # noqa: E731
    return ([('aperture', 'c', 'a', 0.8e-3, 0.8e-3, 0., 0.), ('lens', 10., 10., 0., 0.), ('drift', 10., 0)],
            [pp(), pp(0, tuple(fac)), pp(4)])


def _oracle_electron(args):
    """One macro-electron through the configured beamline with the FP64 oracle (the reference's
    per-electron body: offset field, propagation, total intensity, avg_update_interp order 1 onto
    the common mesh); runs in a spawned process."""
    off, acc = args
    sys.path.insert(0, os.path.join(HERE, 'oracle'))
    import srw_oracle as O
    ex, ey, mesh, sc = synth_undulator_field(1024)
    e2, y2, m2, sc2 = O.electron_offset(ex, ey, mesh, dict(sc, xc=0., yc=0.), *off)
    w = O.Wfr.from_srwl(e2, y2, m2, sc2['Rx'], sc2['Ry'], sc2['dRx'], sc2['dRy'], sc2['xc'], sc2['yc'])
    el, pp = oracle_beamline()
    O.propagate(w, el, pp)
    s = np.zeros((acc['ny'], acc['nx']))
    O.add_interp_bilinear(s, acc, O.total_intensity(w.ex, w.ey), w.out_mesh())
    return s


def _rel_err(a, ref):
    sel = ref > 1e-3 * ref.max()
    return float(np.linalg.norm(a[sel] - ref[sel]) / np.linalg.norm(ref[sel]))


def oracle_error(dev, acc, learned_factors=None):
    """Mean intensity of N_ORACLE electrons of the workload (the bench's offsets and energy spread):
    the batched GPU path with the configured factors and with the learned ones, against the FP64
    oracle run electron by electron with the configured factors; relative L2 where the oracle's
    mean exceeds 1e-3 of its maximum."""
    import multiprocessing as mp
    import torch
    from srw_b200 import srwlib as mod
    from srw_b200.multie import MultiE, sample_offsets
    offs = sample_offsets(N_ORACLE, *SIG, seed=4242, sig_e=SIG_E)
    ex, ey, mesh, sc = synth_undulator_field(1024)
    w = make_wfr(mod, ex, ey, mesh, sc)
    gpu = {}
    for name, fac in (('configured', CONFIGURED), ('learned', learned_factors)):
        if fac is None:
            continue
        me = MultiE(w, beamline_objs(mod, fac), acc, max_batch=N_ORACLE, graph=False, device=dev.index)
        me.add(offs)
        gpu[name] = me.mean()
        del me
    torch.cuda.empty_cache()
    procs = max(1, min(N_ORACLE, os.cpu_count() or 1))
    try:
        import psutil
        procs = max(1, min(procs, int(psutil.virtual_memory().available // ORACLE_PROC_BYTES)))
    except Exception:
        pass
    t0 = time.perf_counter()
    with mp.get_context('spawn').Pool(procs) as pool:
        ref = sum(pool.map(_oracle_electron, [(tuple(o), acc) for o in offs])) / N_ORACLE
    out = {"electrons": N_ORACLE, "oracle": "FP64 numpy restatement (oracle/srw_oracle.py), electron by electron, "
                                            "configured factors (2, 2)", "oracle_processes": procs,
           "oracle_seconds": time.perf_counter() - t0,
           "region": "common-mesh points where the oracle's mean intensity exceeds 1e-3 of its maximum"}
    for name, m in gpu.items():
        out["rel_err_%s_vs_fp64_oracle" % name] = _rel_err(m, ref)
    if learned_factors is not None:
        out["learned_factors"] = list(learned_factors)
    return out


def run_ours(args, rank, world):
    import torch
    import torch.distributed as dist
    from srw_b200 import srwlib as mod
    from srw_b200 import srwlpy as srwl

    dev = torch.device('cuda', int(os.environ.get('LOCAL_RANK', 0)))
    torch.cuda.set_device(dev)
    pl = measure_plain(args, dev, world, dist)
    wm = measure_with_input_moments(args, dev)
    bt = measure_batched(args, dev, world, dist)
    ln = None
    if not args.no_learned:
        ln = measure_learned(args, dev, world, dist, bt['acc'])
    plan, kinfo, per_k = pl['plan'], pl['kinfo'], pl['per_k']
    # the single-wavefront passes at the learned factors (their dominant pass is the headline's)
    pl_l = None
    if ln is not None and not ln['fallback']:
        pl_l = measure_plain(args, dev, world, dist, tuple(ln['factors']))
        ln['plain_at_learned_factors'] = {"ms_per_propagation": pl_l['total_ms'] / pl_l['steps'],
                                          "passes": [list(k) for k in pl_l['kinfo']],
                                          "per_pass_ms": [round(float(v), 4) for v in pl_l['per_k']]}
    peak, peak_src = hbm_peak()
    pass_bytes = sum(kernel_bytes(k) for k in kinfo)
    # algorithmic bytes of one propagation (model: resize reads the old and writes the new mesh,
    # one 2D FFT = one read + one write pass per axis at the new mesh, point-wise work fused; both
    # components): [8 N_in + 8 N_out + 2 * 16 N_out] * 2 = 1,358,954,496 B for 1024^2 -> 4096^2
    n_in, n_out = 1024 * 1024, plan.nx_out * plan.ny_out
    total_alg = (8 * n_in + 8 * n_out + 2 * 16 * n_out) * 2

    # single-wavefront end to end through the drop-in (host buffers in pinned memory)
    e2e_single = None
    if not args.no_e2e:
        e2e_single = e2e_drop_in(args, dev, plan, srwl, mod, world)

    mixed = None
    if not args.no_mixed and world == 1:
        model = None if args.no_learned else load_model(dev)
        mixed = measure_mixed(args, dev, args.mixed_electrons, model)

    if rank != 0:
        return
    orc = None
    if not args.no_oracle:
        lf = tuple(ln['factors']) if (ln is not None and not ln['fallback']) else None
        orc = oracle_error(dev, bt['acc'], lf)
    cpu = None
    if not args.no_cpu_baseline:
        cpu = cpu_baseline_sample(n_props=5)
    if cpu is None:
        why = "not measured (--no-cpu-baseline)" if args.no_cpu_baseline else "reference build not present"
        cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": why}
    # headline: batched + learned factors when the network's factors passed the choice check (no
    # fallback) and, where the oracle leg ran, the learned mean intensity is within 1e-3 of the FP64
    # oracle's on the same electrons; else the batched path with the configured factors
    use_learned = ln is not None and not ln['fallback']
    if use_learned and orc is not None:
        use_learned = orc.get('rel_err_learned_vs_fp64_oracle', 1.) <= 1e-3
    head = ln['value'] if use_learned else bt['value']
    step_batch = LEARNED_BATCH if use_learned else BATCH
    if ln is not None:
        ln['used_for_value'] = use_learned
        ln['vs_plain'] = ln['value'] / pl['value']
    out = {"metric": METRIC, "value": head, "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1000. * step_batch / head, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
           "config": {"workload": WORKLOAD, "step": "one batch of %d macro-electron wavefronts (1024^2 field with "
                                                    "its electron's source offset) through the beamline, intensities "
                                                    "added on the device%s" % (
                                                        step_batch, ", learned factors %s, launched %d electrons "
                                                        "at a time, the mean intensity of the check set checked "
                                                        "against the configured factors before the batch"
                                                        % (ln['factors'], LEARNED_LAUNCH) if use_learned else ""),
                      "grid_in": [1024, 1024], "grid_out": [plan.nx_out, plan.ny_out],
                      "passes": plan.n_kernels, "algorithmic_bytes_per_propagation": total_alg,
                      "pass_bytes_per_propagation": pass_bytes,
                      "l2": "working set per batch >> L2 (126 MB); the plain leg writes a 256 MB buffer between steps",
                      "parallelism": "weak-scaled replicas (independent electrons per rank)" if world > 1 else
                                     "single GPU"},
           "plain": {"value": pl['value'], "unit": UNIT, "ms_per_propagation": pl['total_ms'] / pl['steps'],
                     "steps": pl['steps'], "path": "srwgPlanExecute on a device-resident 1024^2 field, one wavefront "
                                                   "per step"},
           "plain_with_input_moments": wm,
           "batched_vs_plain": bt['value'] / pl['value'],
           "value_vs_plain": head / pl['value'],
           "mean_intensity": {"electrons": bt['n_all'], "peak": bt['mean_peak'],
                              "reduced_over_ranks": world > 1},
           "batched_configured": {"value": bt['value'], "unit": UNIT, "factors": list(CONFIGURED), "batch": BATCH},
           "learned": ln,
           # the dominant pass of the leg that gives `value`, timed inside a batch as it runs there
           "roofline": ln['passes'] if use_learned else bt['passes'],
           "roofline_single_wavefront": roofline(pl_l if (use_learned and pl_l is not None) else pl, peak, peak_src,
                                                 "%s leg, single-wavefront passes, CUDA events per pass" %
                                                 ("learned-factor" if (use_learned and pl_l is not None)
                                                  else "plain")),
           "roofline_plain": dict(roofline(pl, peak, peak_src, "plain leg, CUDA events per pass"),
                                  step_frac=(total_alg / (pl['total_ms'] / pl['steps'] / 1000.) / 1e9) / peak),
           "cpu_baseline": cpu,
           "rel_err_vs_fp64_oracle": (orc or {}).get('rel_err_learned_vs_fp64_oracle' if use_learned else
                                                     'rel_err_configured_vs_fp64_oracle'),
           "oracle_comparison": orc,
           "e2e": (ln['e2e'] if use_learned and ln.get('e2e') else bt['e2e']),
           "e2e_batched_configured": bt['e2e'],
           "e2e_single_wavefront": e2e_single,
           "mixed_grid_multi_electron": mixed,
           "clocks": (ln['clocks'] if use_learned and ln.get('clocks') else bt['clocks']),
           "gpu_launches": (ln['launches_per_step'] if use_learned else plan.n_kernels + 2) * args.steps}
    from srw_b200 import tune
    out["tuning"] = {"table": os.environ.get('SRWG_TUNING', os.path.relpath(tune.TXT, HERE)),
                     "headline": tune.pass_shapes(ln['passes']['passes']) if use_learned else None,
                     "plain": tune.pass_shapes(plan.kernels())}
    print(json.dumps(out))


def roofline(pl, peak, peak_src, where):
    """Roofline object of the dominant pass of a measure_plain result: algorithmic bytes per launch
    over its average CUDA-event time, against the HBM peak."""
    kinfo, per_k = pl['kinfo'], pl['per_k']
    kd = int(np.argmax(per_k))
    alg = kernel_bytes(kinfo[kd])
    achieved = alg / (per_k[kd] / 1000.) / 1e9
    return {"bound": "hbm", "kernel": "%s %s" % (kinfo[kd][0], 'x'.join(map(str, kinfo[kd][1:]))),
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_src,
            "traffic": TRAFFIC.get(kinfo[kd]), "algorithmic_bytes": alg, "avg_ms": float(per_k[kd]),
            "per_pass_ms": [round(float(v), 4) for v in per_k], "passes": [list(k) for k in kinfo],
            "measured_on": where}


def e2e_drop_in(args, dev, plan, srwl, mod, world):
    """The single-wavefront drop-in srwlpy.PropagElecField with pinned host buffers: H2D of the
    input and D2H of the 4096^2 result inside the timed region."""
    import torch
    ex, ey, mesh, sc = synth_undulator_field(1024)
    pinned = []

    def palloc(n):
        t = torch.empty(n, dtype=torch.float32).pin_memory()
        pinned.append(t)
        return t.numpy()

    class PinnedWfr(mod.SRWLWfr):
        def allocate(self, _ne, _nx, _ny, _EXNeeded=1, _EYNeeded=1, _typeE='f', _backupNeeded=0):
            mod.SRWLWfr.allocate(self, _ne, 0, 0, _EXNeeded, _EYNeeded, _typeE, _backupNeeded)
            if _EXNeeded:
                self.arEx = out_bufs[0]
            if _EYNeeded:
                self.arEy = out_bufs[1]
            self.mesh.nx, self.mesh.ny = _nx, _ny

    out_bufs = [palloc(2 * plan.nx_out * plan.ny_out), palloc(2 * plan.nx_out * plan.ny_out)]
    in_x, in_y = palloc(2 * ex.size), palloc(2 * ey.size)
    in_x[0::2], in_x[1::2] = ex.real.ravel(), ex.imag.ravel()
    in_y[0::2], in_y[1::2] = ey.real.ravel(), ey.imag.ravel()
    bl = beamline_objs(mod)

    def once():
        wp = PinnedWfr()
        wp.allocate(1, 1024, 1024)
        wp.arEx, wp.arEy = in_x, in_y
        for k in ('xStart', 'xFin', 'yStart', 'yFin', 'eStart', 'eFin', 'zStart'):
            setattr(wp.mesh, k, mesh[k])
        wp.Rx, wp.Ry, wp.dRx, wp.dRy = sc['Rx'], sc['Ry'], sc['dRx'], sc['dRy']
        srwl.PropagElecField(wp, bl, None, dev.index + 1)
        return wp

    for _ in range(2):
        once()
    n_e2e = max(3, min(args.steps, 10))
    t0 = time.perf_counter()
    for _ in range(n_e2e):
        wp = once()
        _ = float(wp.arEx[0])                              # host read of the result
    e2e_s = time.perf_counter() - t0
    return {"value": world * n_e2e / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 2 * 8 * 1024 * 1024,
            "d2h_bytes_per_step": 2 * 8 * plan.nx_out * plan.ny_out,
            "path": "srw_b200.srwlpy.PropagElecField (C-ABI srwlPropagElecField), pinned host buffers"}


def spawn_ranks(n):
    """`--gpus N` without a launcher: runs this script under torch.distributed.run with N ranks on
    this node (rendezvous on 127.0.0.1), bounded by an outer timeout; returns its exit code."""
    import socket
    with socket.socket() as sk:
        sk.bind(('127.0.0.1', 0))
        port = sk.getsockname()[1]
    cmd = ['timeout', '-k', '60', '3600', sys.executable, '-m', 'torch.distributed.run', '--nnodes=1',
           '--nproc-per-node', str(n), '--master-addr', '127.0.0.1', '--master-port', str(port),
           os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=200)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-e2e', action='store_true', help='skip the end-to-end legs (profiling runs)')
    ap.add_argument('--no-mixed', action='store_true', help='skip the mixed-grid multi-electron workload')
    ap.add_argument('--no-learned', action='store_true', help='skip the learned-factor leg')
    ap.add_argument('--mixed-electrons', type=int, default=2000)
    ap.add_argument('--no-oracle', action='store_true', help='skip the FP64-oracle error leg')
    args = ap.parse_args()
    if args.gpus > 1 and 'WORLD_SIZE' not in os.environ:
        sys.exit(spawn_ranks(args.gpus))
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    if args.impl == 'reference':
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get('LOCAL_RANK', 0)))
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=120))
    try:
        run_ours(args, rank, world)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == '__main__':
    main()
