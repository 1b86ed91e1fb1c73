"""Small, fixed workloads of the undulator beamline for kernel profiles (ncu) and launch lists.

    python -m srw_b200.profile_cases batch --factors 1,2,1.25,1.5 --batch 8 --batches 3
    python -m srw_b200.profile_cases plain --factors 2,2,2,2 --reps 3

`batch`: macro-electron batches (srw_b200.multie.MultiE, no graph: every pass is its own launch) of
the 1024^2 undulator-like field through aperture -> resize (factors) -> lens -> drift to the waist,
intensities added on a 512^2 detector mesh; `plain`: single-wavefront propagations (srwgPlanExecute)
of the same field.  The field and the electrons are the bench's (bench.synth_undulator_field,
bench.SIG).  Prints the passes of the plan.
"""
import argparse
import os
import sys


def main():
    import torch
    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, here)
    import bench
    from srw_b200 import srwlib as mod
    from srw_b200.multie import MultiE, sample_offsets
    from srw_b200.plan import Plan
    ap = argparse.ArgumentParser()
    ap.add_argument('what', choices=['batch', 'plain'])
    ap.add_argument('--factors', default='2,2,2,2')
    ap.add_argument('--batch', type=int, default=8)
    ap.add_argument('--batches', type=int, default=3)
    ap.add_argument('--reps', type=int, default=3)
    a = ap.parse_args()
    fac = tuple(float(v) for v in a.factors.split(','))
    ex, ey, mesh, sc = bench.synth_undulator_field(1024)
    w = bench.make_wfr(mod, ex, ey, mesh, sc)
    dev = torch.device('cuda', 0)
    if a.what == 'batch':
        acc = bench._acc_mesh(Plan(w, bench.beamline_objs(mod), device=0))
        me = MultiE(w, bench.beamline_objs(mod, fac), acc, max_batch=a.batch, graph=False, device=0)
        for k in range(a.batches):
            me.add(sample_offsets(a.batch, *bench.SIG, seed=5, first=a.batch * k, sig_e=bench.SIG_E))
        torch.cuda.synchronize(dev)
        print(me.info())
    else:
        p = Plan(w, bench.beamline_objs(mod, fac), device=0)
        dex, dey = torch.from_numpy(ex).to(dev), torch.from_numpy(ey).to(dev)
        ox, oy = p.new_output()
        for _ in range(a.reps):
            p.execute(dex, dey, ox, oy)
        torch.cuda.synchronize(dev)
        print(p.describe())


if __name__ == '__main__':
    main()
