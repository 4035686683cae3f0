"""Server-side voxeliser: the browser's voxelize.js (web/js/voxelize.js:5-115) run on the GPU
through wt_voxelize, so an uploaded triangle soup in lattice coordinates becomes the solid mask
Solver.set_solid takes, with the frontal and planform areas the client uses for Cd/Cl.
"""
import ctypes

import numpy as np
import torch

import wtlib as W
from wtlib import ptr


def voxelize(tris, dims, ground=True, device='cuda:0', stream=None):
    """tris: (T, 9) lattice-space triangle corners (float32). Returns (solid uint8 numpy (n,),
    dict(frontal, planform, count, crossings)) as voxelize.js returns them."""
    nx, ny, nz = (int(d) for d in dims)
    dev = torch.device(device)
    st = stream if stream is not None else torch.cuda.current_stream(dev)
    sh = W.stream_handle(st)
    host = np.ascontiguousarray(np.asarray(tris, np.float32).reshape(-1, 9))
    with torch.cuda.stream(st):
        t = torch.from_numpy(host).to(dev) if len(host) else torch.zeros((1, 9), dtype=torch.float32, device=dev)
        solid = torch.empty(nx * ny * nz, dtype=torch.uint8, device=dev)
    out = (ctypes.c_int64 * 4)()
    cap = max(4096, 4 * ny * nz)
    for _ in range(2):
        nbytes = int(W.lib().wt_voxelize_workspace_bytes(nx, ny, nz, cap))
        if nbytes < 0:
            W.check(nbytes)
        with torch.cuda.stream(st):
            ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        rc = W.lib().wt_voxelize(ptr(t), len(host), nx, ny, nz, 1 if ground else 0, ptr(solid), ptr(ws), nbytes,
                                 out, sh)
        if rc == W.WT_ERR_CAPACITY and out[3] > cap:
            cap = int(out[3])  # one more pass with room for every crossing
            continue
        W.check(rc)
        break
    return solid.cpu().numpy(), dict(frontal=int(out[0]), planform=int(out[1]), count=int(out[2]),
                                     crossings=int(out[3]))
