"""Storage-precision accuracy study against an FP64 run of the identical tunnel.

Runs the same tunnel (default: the 6-ellipsoid body on a moving belt scaled to
256x128x128, u = 0.05, nu = 0.001, Cs = 0.16; `nu` selects another viscosity) for `steps`
steps in FP64 (reference-order
collision, itself bit-identical to the CPU oracle in fp64) and in each candidate form, then
reports against the FP64 run:
  * velocity relative L2 error over fluid cells, ||u - u64|| / ||u64||,
  * pressure max-abs error, p = (rho - 1) / 3, over fluid cells,
  * both for the last step's fields and for the fields averaged over the last `avg_window`
    steps (every step, or every `field_every` steps), and the instantaneous velocity error at
    checkpoint steps;
  * drag and lift coefficients Cd = Fx / (0.5 u^2 A), Cl = Fy / (0.5 u^2 A) (A = frontal
    area of the body, web/js/main.js:337-339), instantaneous at the last step and averaged
    over the last `avg_window` steps (forces sampled every `sample_every` steps), relative
    error of Cd and absolute error of Cl (Cl of a near-symmetric body is close to 0).

At nu = 0.001 the wake is chaotic: any change of rounding (fp32 against fp64 included)
grows into a different instantaneous flow within the run, so the late instantaneous figures
bound nothing but the statistics; the checkpoint errors show the growth, and fp32's errors
are the floor no storage precision can go below. Statistics need a window of several vortex
shedding periods after the wake has formed: `long_study` runs 40,000 steps (about eight
flow-through times of the 256-cell tunnel) and averages over the last 30,000. At nu = 0.02
(Re about 100 on the body) the flow is laminar and the differences measure the storage
precision itself.

    python wind-tunnel_b200/accuracy.py [--steps 2000] [--scale 0.5] [--nu 0.001]
"""
import argparse
import json
import os
import sys

import numpy as np
import torch

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import bodies  # noqa: E402
import lbm  # noqa: E402

CANDIDATES = [('fp32', 'exact'), ('fp32', 'fast'), ('fp16', 'fast'), ('bf16', 'fast'), ('fp16', 'exact')]


CHECKPOINTS = (100, 500, 1000, 2000)
LONG_CHECKPOINTS = (100, 500, 1000, 2000, 5000, 10000, 20000)


def run(dims, solid, p, precision, collision, steps, sample_every, avg_window, device, checkpoints=CHECKPOINTS,
        field_every=1):
    """One tunnel for `steps` steps. Returns the last step's mac, its drag and lift (fp64 sums
    without the y = 0 plane), their means over the last `avg_window` steps (sampled every
    `sample_every` steps), mac time-averaged over the last `avg_window` steps (every
    `field_every`-th step, in fp64 on the device) and mac at each checkpoint step."""
    avg_window = max(1, min(avg_window, steps))
    field_every = max(1, min(field_every, sample_every))
    assert sample_every % field_every == 0, 'forces are sampled on field steps'
    s = lbm.Solver(dims, device, precision=precision, collision=collision)
    s.set_solid(solid)
    s.reset(p['uIn'])
    fx, fy = [], []
    snaps = {}
    acc = torch.zeros((s.n, 4), dtype=torch.float64, device=s.dev)
    stops = sorted({c for c in checkpoints if c < steps} | {steps - avg_window, steps})
    done, fields = 0, 0
    while done < steps:
        if done >= steps - avg_window:  # inside the averaging window: field_every steps at a time
            k = min(field_every, steps - done)
            s.step(k, p)
            done += k
            s.synchronize()
            acc += s.mac[s.cur].double()
            fields += 1
            if (done - (steps - avg_window)) % sample_every == 0:
                f6 = s.forces6()
                fx.append(f6[3])
                fy.append(f6[4])
        else:
            k = min(sample_every, next(c for c in stops if c > done) - done)
            s.step(k, p)
            done += k
        if done in checkpoints and done < steps:
            snaps[done] = s.macro()
    mac = s.macro()
    snaps[steps] = mac
    f6 = s.forces6()
    mean_mac = (acc / max(1, fields)).cpu().numpy()
    del s, acc
    torch.cuda.empty_cache()
    return mac, (f6[3], f6[4]), (float(np.mean(fx)), float(np.mean(fy))), mean_mac, snaps


def _field_errors(mac, ref, fluid):
    u, u_ref = mac[fluid, :3], ref[fluid, :3]
    pr, p_ref = (mac[fluid, 3] - 1.0) / 3.0, (ref[fluid, 3] - 1.0) / 3.0
    return float(np.linalg.norm(u - u_ref) / np.linalg.norm(u_ref)), float(np.abs(pr - p_ref).max())


def study(steps=2000, scale=0.5, device='cuda:0', sample_every=10, avg_window=500, candidates=CANDIDATES, nu=None,
          field_every=1, checkpoints=CHECKPOINTS):
    """Every candidate form against the FP64 run: instantaneous fields, drag and lift at the last
    step; the same averaged over the last `avg_window` steps; the instantaneous velocity error
    at each checkpoint (how it grows from the storage rounding). In a chaotic regime the fp32
    form's errors are the floor that storage precision cannot go below."""
    dims, solid, p = bodies.config2(scale=scale)
    if nu is not None:
        p['tau'] = 3.0 * nu + 0.5
    nu_used = (p['tau'] - 0.5) / 3.0
    avg_window = max(1, min(avg_window, steps))
    frontal, _ = bodies.areas(solid, dims)
    q = 0.5 * p['uIn'] ** 2 * max(1, frontal)
    fluid = solid == 0
    ref_mac, ref_f, ref_avg, ref_mean, ref_snaps = run(dims, solid, p, 'fp64', 'exact', steps, sample_every,
                                                       avg_window, device, checkpoints, field_every)
    cd_ref, cl_ref = ref_f[0] / q, ref_f[1] / q
    cd_ref_avg, cl_ref_avg = ref_avg[0] / q, ref_avg[1] / q
    out = {'workload': f'{dims[0]}x{dims[1]}x{dims[2]}, 6-ellipsoid body on moving belt, u = {p["uIn"]}, '
                       f'nu = {nu_used:.4g}, {steps} steps',
           'reference': 'fp64 storage and arithmetic, reference-order collision',
           'averaging': (f'fields averaged over the last {avg_window} steps, every '
                         f'{"" if field_every == 1 else f"{field_every}th "}step; Cd/Cl over the same window '
                         f'every {sample_every} steps'),
           'cd_fp64': cd_ref, 'cl_fp64': cl_ref, 'cd_fp64_avg': cd_ref_avg, 'cl_fp64_avg': cl_ref_avg,
           'frontal_area_cells': frontal, 'forms': {}}
    for precision, collision in candidates:
        mac, f, avg, mean, snaps = run(dims, solid, p, precision, collision, steps, sample_every, avg_window, device,
                                       checkpoints, field_every)
        vel, pres = _field_errors(mac, ref_mac, fluid)
        avel, apres = _field_errors(mean, ref_mean, fluid)
        cd, cl = f[0] / q, f[1] / q
        cda, cla = avg[0] / q, avg[1] / q
        out['forms'][f'{precision}-{collision}'] = {
            'velocity_rel_l2': vel, 'pressure_max_abs': pres,
            'cd': cd, 'cd_rel_err': abs(cd - cd_ref) / abs(cd_ref), 'cl_abs_err': abs(cl - cl_ref),
            'avg_velocity_rel_l2': avel, 'avg_pressure_max_abs': apres,
            'cd_avg_rel_err': abs(cda - cd_ref_avg) / abs(cd_ref_avg), 'cl_avg_abs_err': abs(cla - cl_ref_avg),
            'velocity_rel_l2_at': {str(k): _field_errors(snaps[k], ref_snaps[k], fluid)[0]
                                   for k in sorted(snaps) if k in ref_snaps},
        }
    return out


def long_study(device='cuda:0', steps=40000, avg_window=30000, scale=0.5):
    """The chaotic regime's statistics: 40,000 steps at nu = 0.001 with fields and forces
    averaged every 10 steps over the last 30,000."""
    return study(steps=steps, scale=scale, device=device, sample_every=10, avg_window=avg_window, field_every=10,
                 checkpoints=LONG_CHECKPOINTS)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--steps', type=int, default=2000)
    ap.add_argument('--scale', type=float, default=0.5)
    ap.add_argument('--nu', type=float, default=None)
    ap.add_argument('--long', action='store_true', help='the 40,000-step statistics regime')
    a = ap.parse_args()
    print(json.dumps(long_study(scale=a.scale) if a.long else study(a.steps, a.scale, nu=a.nu)), flush=True)


if __name__ == '__main__':
    main()
