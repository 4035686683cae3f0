"""Storage-precision accuracy study against an FP64 run of the identical tunnel.

Runs the same tunnel (default: the 6-ellipsoid body on a moving belt scaled to
256x128x128, u = 0.05, nu = 0.001, Cs = 0.16; `nu` selects another viscosity) for `steps`
steps in FP64 (reference-order
collision, itself bit-identical to the CPU oracle in fp64) and in each candidate form, then
reports against the FP64 run:
  * velocity relative L2 error over fluid cells, ||u - u64|| / ||u64||,
  * pressure max-abs error, p = (rho - 1) / 3, over fluid cells,
  * drag and lift coefficients Cd = Fx / (0.5 u^2 A), Cl = Fy / (0.5 u^2 A) (A = frontal
    area of the body), instantaneous at the last step and averaged over the last
    `avg_window` steps (forces sampled every `sample_every` steps), relative error of Cd
    and absolute error of Cl (Cl of a near-symmetric body is close to 0).

At nu = 0.001 the wake is chaotic: any change of rounding (fp32 against fp64 included)
grows into a different instantaneous flow within the run, so those figures bound nothing
but the statistics. At nu = 0.02 (Re about 100 on the body) the flow is laminar and the
differences measure the storage precision itself.

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


def run(dims, solid, p, precision, collision, steps, sample_every, avg_window, device):
    s = lbm.Solver(dims, device, precision=precision, collision=collision)
    s.set_solid(solid)
    s.reset(p['uIn'])
    fx, fy = [], []
    done = 0
    while done < steps:
        k = min(sample_every, steps - done)
        s.step(k, p)
        done += k
        if done > steps - avg_window:
            f6 = s.forces6()
            fx.append(f6[3])
            fy.append(f6[4])
    mac = s.macro()
    f6 = s.forces6()
    del s
    torch.cuda.empty_cache()
    return mac, (f6[3], f6[4]), (float(np.mean(fx)), float(np.mean(fy)))


def study(steps=2000, scale=0.5, device='cuda:0', sample_every=10, avg_window=500, candidates=CANDIDATES, nu=None):
    dims, solid, p = bodies.config2(scale=scale)
    if nu is not None:
        p['tau'] = 3.0 * nu + 0.5
    nu_used = (p['tau'] - 0.5) / 3.0
    frontal, _ = bodies.areas(solid, dims)
    q = 0.5 * p['uIn'] ** 2 * max(1, frontal)
    fluid = solid == 0
    ref_mac, ref_f, ref_avg = run(dims, solid, p, 'fp64', 'exact', steps, sample_every, avg_window, device)
    u_ref = ref_mac[fluid, :3]
    p_ref = (ref_mac[fluid, 3] - 1.0) / 3.0
    cd_ref, cl_ref = ref_f[0] / q, ref_f[1] / q
    cd_ref_avg, cl_ref_avg = ref_avg[0] / q, ref_avg[1] / q
    out = {'workload': f'{dims[0]}x{dims[1]}x{dims[2]}, 6-ellipsoid body on moving belt, u = {p["uIn"]}, '
                       f'nu = {nu_used:.4g}, {steps} steps',
           'reference': 'fp64 storage and arithmetic, reference-order collision',
           'cd_fp64': cd_ref, 'cl_fp64': cl_ref, 'cd_fp64_avg': cd_ref_avg, 'cl_fp64_avg': cl_ref_avg,
           'frontal_area_cells': frontal, 'forms': {}}
    for precision, collision in candidates:
        mac, f, avg = run(dims, solid, p, precision, collision, steps, sample_every, avg_window, device)
        u = mac[fluid, :3]
        pr = (mac[fluid, 3] - 1.0) / 3.0
        cd, cl = f[0] / q, f[1] / q
        cda, cla = avg[0] / q, avg[1] / q
        out['forms'][f'{precision}-{collision}'] = {
            'velocity_rel_l2': float(np.linalg.norm(u - u_ref) / np.linalg.norm(u_ref)),
            'pressure_max_abs': float(np.abs(pr - p_ref).max()),
            'cd': cd, 'cd_rel_err': abs(cd - cd_ref) / abs(cd_ref), 'cl_abs_err': abs(cl - cl_ref),
            'cd_avg_rel_err': abs(cda - cd_ref_avg) / abs(cd_ref_avg), 'cl_avg_abs_err': abs(cla - cl_ref_avg),
        }
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--steps', type=int, default=2000)
    ap.add_argument('--scale', type=float, default=0.5)
    ap.add_argument('--nu', type=float, default=None)
    a = ap.parse_args()
    print(json.dumps(study(a.steps, a.scale, nu=a.nu)), flush=True)


if __name__ == '__main__':
    main()
