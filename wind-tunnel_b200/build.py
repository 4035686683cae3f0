"""Build libwt.so (sm_100a) in-tree from csrc/*.cu with nvcc.

The library is compiled without FMA contraction (-fmad=false) and with IEEE division and
square root (nvcc's defaults), so every kernel evaluates the reference's float expressions
in the reference's order and matches the oracle bit for bit.

    python wind-tunnel_b200/build.py          # builds wind-tunnel_b200/libwt.so
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
OUT = os.path.join(HERE, 'libwt.so')
# the step and batch kernels are instantiated once per storage precision (wt_kernels_<prec>.cu),
# the largest sources first so the parallel build finishes soonest
SOURCES = ['wt_kernels_f64.cu', 'wt_kernels_f32.cu', 'wt_kernels_f16.cu', 'wt_kernels_bf16.cu', 'wt_abi.cu',
           'wt_setup.cu', 'wt_step.cu', 'wt_batch.cu', 'wt_reduce.cu', 'wt_frame.cu', 'wt_voxel.cu']
NVCC = os.environ.get('NVCC', '/usr/local/cuda/bin/nvcc')
FLAGS = ['-gencode', 'arch=compute_100a,code=sm_100a', '-lineinfo', '-O3', '-std=c++17', '-fmad=false',
         '-Xcompiler', '-fPIC', '-Xcompiler', '-O2', '--ptxas-options=-v', '-ccbin', 'g++']


def _newest(paths):
    return max(os.path.getmtime(p) for p in paths)


def build(force=False, verbose=False):
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith('.cuh')]
    deps.append(os.path.join(HERE, '..', 'include', 'wt.h'))
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= _newest(deps):
        return OUT
    objdir = os.path.join(HERE, '_build')
    os.makedirs(objdir, exist_ok=True)
    objs = [os.path.join(objdir, os.path.basename(s).replace('.cu', '.o')) for s in srcs]

    def compile_one(src_obj):
        src, obj = src_obj
        return src, subprocess.run([NVCC, *FLAGS, '-c', src, '-o', obj], capture_output=True, text=True)

    jobs = max(1, min(len(srcs), os.cpu_count() or 1))
    with ThreadPoolExecutor(jobs) as pool:
        for src, r in pool.map(compile_one, zip(srcs, objs)):
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise RuntimeError(f'nvcc failed on {src}')
            if verbose:
                sys.stderr.write(r.stderr)
    tmp = OUT + '.tmp'
    r = subprocess.run([NVCC, '-gencode', 'arch=compute_100a,code=sm_100a', '-shared', '-o', tmp, *objs],
                       capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError('nvcc link failed')
    os.replace(tmp, OUT)
    return OUT


if __name__ == '__main__':
    print(build(force='--force' in sys.argv, verbose='-v' in sys.argv))
