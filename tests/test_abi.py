"""The C-ABI library loads, exports every symbol include/wt.h declares, and rejects bad
arguments with its error codes -- all without touching a GPU."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

import wtlib as W


@pytest.fixture(scope='module')
def L():
    import build
    build.build()
    return W.lib()


def _declared():
    names = set()
    for h in os.listdir(os.path.join(ROOT, 'include')):
        if h.endswith('.h'):
            txt = open(os.path.join(ROOT, 'include', h)).read()
            names |= set(re.findall(r'^\s*(?:const\s+)?[\w\s\*]+?\b(wt_\w+)\s*\(', txt, re.M))
    return names


def test_header_declares_what_binding_binds():
    assert _declared() == set(W.EXPORTS)


def test_exports_every_declared_symbol(L):
    for name in _declared():
        assert hasattr(L, name), name


def test_abi_version(L):
    assert L.wt_abi_version() == W.ABI_VERSION == 4


@pytest.mark.parametrize('dims,ok', [((128, 64, 64), True), ((4, 3, 3), True), ((12, 8, 10), True),
                                     ((3, 8, 8), False), ((13, 8, 8), False), ((16, 2, 8), False),
                                     ((16, 8, 2), False), ((2048, 2048, 1024), False)])
def test_check_dims(L, dims, ok):
    rc = L.wt_check_dims(*dims)
    assert (rc == 0) == ok
    if not ok:
        assert rc == W.WT_ERR_DIMS
        assert b'grid' in L.wt_last_error()


def test_population_bytes(L):
    assert L.wt_population_bytes(W.F32, 100) == 7600
    assert L.wt_population_bytes(W.F16, 100) == 3800
    assert L.wt_population_bytes(W.BF16, 100) == 3800
    assert L.wt_population_bytes(W.F64, 100) == 15200
    assert L.wt_population_bytes(9, 100) == -1


def test_null_arguments_rejected_before_any_launch(L):
    assert L.wt_step(None, 0, 1, 0.05, 0.506, 0.16, 1, None) == W.WT_ERR_ARG
    assert b'null' in L.wt_last_error()
    g = W.Grid(16, 8, 8, W.F32)
    assert L.wt_step(ctypes.byref(g), 0, 1, 0.05, 0.5, 0.1, 1, None) == W.WT_ERR_ARG
    assert L.wt_init_eq(W.F32, None, None, 10, 0.05, 0.0, None) == W.WT_ERR_ARG
    assert L.wt_forces(None, 0, None, None, 0, None, None, None) == W.WT_ERR_ARG
    assert L.wt_mass(None, 0, None, None, None) == W.WT_ERR_ARG
    assert L.wt_slice(None, None, None, 16, 8, 8, 0, 0, 0, 0.05, 1.0, 0.0, 1.0, None) == W.WT_ERR_ARG
    assert L.wt_links_scan(None, None, None, None) == W.WT_ERR_ARG


def test_bad_enums_rejected(L):
    fake = ctypes.c_void_p(16)  # never dereferenced: validation fails first
    g = W.Grid(16, 8, 8, 7, (ctypes.c_void_p * 2)(16, 16), (ctypes.c_void_p * 2)(16, 16), 16, 16)
    assert L.wt_step(ctypes.byref(g), 0, 1, 0.05, 0.5, 0.1, 1, None) == W.WT_ERR_ARG
    assert b'precision' in L.wt_last_error()
    g.precision = W.F32
    assert L.wt_step(ctypes.byref(g), 2, 1, 0.05, 0.5, 0.1, 1, None) == W.WT_ERR_ARG
    assert L.wt_init_eq(9, fake, fake, 10, 0.05, 0.0, None) == W.WT_ERR_ARG
    g.nx = 15
    assert L.wt_step(ctypes.byref(g), 0, 1, 0.05, 0.5, 0.1, 1, None) == W.WT_ERR_DIMS
    g.nx = 16
    assert L.wt_step(ctypes.byref(g), 0, 0, 0.05, 0.5, 0.1, 1, None) == W.WT_OK  # zero steps: no launch
    assert L.wt_slice(fake, fake, fake, 16, 8, 8, 5, 0, 0, 0.05, 1.0, 0.0, 1.0, None) == W.WT_ERR_ARG
    assert L.wt_slice(fake, fake, fake, 16, 8, 8, 1, 8, 0, 0.05, 1.0, 0.0, 1.0, None) == W.WT_ERR_ARG


def test_scratch_sizes(L):
    assert L.wt_links_scratch_len(1024) == 2
    assert L.wt_links_scratch_len(1025) == 3
    assert L.wt_reduce_scratch_len(10) >= 6
