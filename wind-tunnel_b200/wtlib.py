"""ctypes binding of libwt.so (declared in include/wt.h).

This is the thin C-ABI layer between the Python host code and the sm_100a kernels. Device
buffers are torch tensors used only as memory (their ``data_ptr()``); streams are passed
as raw ``cudaStream_t`` handles. There is no fallback: if ``libwt.so`` is missing or
fails to load, ``lib()`` raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, 'libwt.so')

WT_OK, WT_ERR_ARG, WT_ERR_DIMS, WT_ERR_CUDA, WT_ERR_CAPACITY, WT_ERR_TIMEOUT = 0, -1, -2, -3, -4, -5
F32, F16, BF16, F64 = 0, 1, 2, 3
PRECISIONS = {'fp32': F32, 'fp16': F16, 'bf16': BF16, 'fp64': F64}
STEP_MAC_ALL_LAST = 1
NOALLOC_MAX_LINKS = 1048576  # wt_forces_noalloc limit (include/wt.h)
COLLIDE_EXACT, COLLIDE_FAST = 0, 1

# every symbol include/wt.h declares (tests check that the library exports them all)
EXPORTS = ['wt_last_error', 'wt_abi_version', 'wt_check_dims', 'wt_population_bytes', 'wt_init_eq',
           'wt_build_codes', 'wt_links_scratch_len', 'wt_links_scan', 'wt_links_fill', 'wt_step_tiles', 'wt_step',
           'wt_step_test_skip_chunk',
           'wt_reduce_scratch_len', 'wt_forces', 'wt_forces_noalloc', 'wt_mass', 'wt_batch_workspace_bytes',
           'wt_batch_create', 'wt_batch_step', 'wt_batch_step_each', 'wt_batch_capture', 'wt_batch_replay', 'wt_batch_cur',
           'wt_batch_destroy', 'wt_advect', 'wt_pack_particles', 'wt_slice', 'wt_cp',
           'wt_voxelize_workspace_bytes', 'wt_voxelize']


class WtError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f'libwt error {code}: {msg}')
        self.code = code


class Grid(ctypes.Structure):
    """struct wt_grid (include/wt.h)."""
    _fields_ = [('nx', ctypes.c_int32), ('ny', ctypes.c_int32), ('nz', ctypes.c_int32),
                ('precision', ctypes.c_int32),
                ('f', ctypes.c_void_p * 2), ('mac', ctypes.c_void_p * 2),
                ('solid', ctypes.c_void_p), ('code', ctypes.c_void_p),
                ('tile', ctypes.c_int32), ('collision', ctypes.c_int32),
                ('status', ctypes.c_void_p), ('shift_u', ctypes.c_float)]


_lib = None
ABI_VERSION = 4  # include/wt.h WT_ABI_VERSION this binding is written against


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f'libwt.so not built ({LIB_PATH}); run wind-tunnel_b200/build.py')
        L = ctypes.CDLL(LIB_PATH)
        vp, i32, i64, u32, f32, f64 = (ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_uint32,
                                       ctypes.c_float, ctypes.c_double)
        gp = ctypes.POINTER(Grid)
        sig = {
            'wt_last_error': ([], ctypes.c_char_p),
            'wt_abi_version': ([], ctypes.c_int),
            'wt_check_dims': ([i32, i32, i32], ctypes.c_int),
            'wt_population_bytes': ([i32, i64], i64),
            'wt_init_eq': ([i32, vp, vp, i64, f64, f64, vp], ctypes.c_int),
            'wt_build_codes': ([gp, vp], ctypes.c_int),
            'wt_links_scratch_len': ([i64], i64),
            'wt_links_scan': ([gp, vp, vp, vp], ctypes.c_int),
            'wt_links_fill': ([gp, vp, vp, vp, i64, vp], ctypes.c_int),
            'wt_step_tiles': ([i32, i32, vp, i32], ctypes.c_int),
            'wt_step': ([gp, i32, i32, f64, f64, f64, i32, vp], ctypes.c_int),
            'wt_step_test_skip_chunk': ([gp, i32, i32, f64, f64, f64, i32, i32, vp], ctypes.c_int),
            'wt_reduce_scratch_len': ([i64], i64),
            'wt_forces': ([gp, i32, vp, vp, i64, vp, vp, vp], ctypes.c_int),
            'wt_forces_noalloc': ([gp, i32, vp, vp, i64, vp, vp], ctypes.c_int),
            'wt_mass': ([gp, i32, vp, vp, vp], ctypes.c_int),
            'wt_batch_workspace_bytes': ([gp, i32, i32], i64),
            'wt_batch_create': ([gp, i32, vp, vp, vp, vp, i32, vp, i64, vp, ctypes.POINTER(vp)], ctypes.c_int),
            'wt_batch_step': ([vp, i32, i32, vp], ctypes.c_int),
            'wt_batch_step_each': ([vp, vp, i32, vp], ctypes.c_int),
            'wt_batch_capture': ([vp, i32, i32, vp], ctypes.c_int),
            'wt_batch_replay': ([vp, vp], ctypes.c_int),
            'wt_batch_cur': ([vp, vp], ctypes.c_int),
            'wt_batch_destroy': ([vp], ctypes.c_int),
            'wt_advect': ([vp, vp, vp, vp, i32, i32, i32, i64, f32, f32, f32, u32, f32, f32, f32, f32, f32, vp],
                          ctypes.c_int),
            'wt_pack_particles': ([vp, vp, vp, vp, i32, i32, i32, i64, vp], ctypes.c_int),
            'wt_slice': ([vp, vp, vp, i32, i32, i32, i32, i32, i32, f32, f32, f32, f32, vp], ctypes.c_int),
            'wt_cp': ([vp, vp, vp, vp, vp, i32, i32, i32, i64, f32, f32, vp], ctypes.c_int),
            'wt_voxelize_workspace_bytes': ([i32, i32, i32, i64], ctypes.c_int64),
            'wt_voxelize': ([vp, i64, i32, i32, i32, i32, vp, vp, i64, vp, vp], ctypes.c_int),
        }
        for name, (args, res) in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        if L.wt_abi_version() != ABI_VERSION:
            raise RuntimeError(f'libwt.so ABI {L.wt_abi_version()} != {ABI_VERSION}; rebuild wind-tunnel_b200')
        _lib = L
    return _lib


def check(rc):
    if rc != WT_OK:
        raise WtError(rc, lib().wt_last_error().decode(errors='replace'))
    return rc


def call(name, *args):
    return check(getattr(lib(), name)(*args))


def ptr(t):
    """Raw device (or host) address of a tensor, or None."""
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def step_tiles(precision, collision=COLLIDE_EXACT):
    """[(id, cells_per_thread, threads_per_block, min_blocks_per_sm), ...] of the step kernel for
    a storage precision and collision form (COLLIDE_EXACT / COLLIDE_FAST, or 'exact' / 'fast')."""
    if isinstance(collision, str):
        collision = {'exact': COLLIDE_EXACT, 'fast': COLLIDE_FAST}[collision]
    buf = (ctypes.c_int32 * 256)()
    n = lib().wt_step_tiles(int(precision), int(collision), buf, 64)
    if n < 0:
        check(n)
    return [tuple(buf[4 * k:4 * k + 4]) for k in range(n)]


def stream_handle(stream):
    return ctypes.c_void_p(stream.cuda_stream if stream is not None else 0)
