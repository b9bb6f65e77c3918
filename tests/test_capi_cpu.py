"""C ABI checks that need no GPU: the library loads, exports every entry point
include/hodlr_gpu.h declares, builds the reference's tree, and rejects bad
arguments before touching a device."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, cuda_available


def declared_functions():
    txt = open(os.path.join(ROOT, "include", "hodlr_gpu.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = re.findall(r"\b(hodlr_[a-z0-9_]+)\s*\(", txt)
    return sorted(set(names))


def test_header_declares_the_task_bodies():
    names = declared_functions()
    for fn in ["hodlr_leaf_solve", "hodlr_gemm_reduce", "hodlr_node_lu_solve",
               "hodlr_node_schur2_solve", "hodlr_gemm_broadcast", "hodlr_leaf_solve_batched",
               "hodlr_create", "hodlr_solve_fused", "hodlr_factor", "hodlr_solve",
               "hodlr_solve_refined", "hodlr_matvec"]:
        assert fn in names


def test_library_exports_every_declared_symbol(fs):
    lib = ctypes.CDLL(fs.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


@pytest.mark.parametrize("args", [(480, 2, 30, 60), (4096, 1, 30, 256), (1025, 3, 7, 100),
                                  (201, 3, 10, 100), (262144, 16, 64, 512),
                                  (65536, 8, 50, 512), (100003, 7, 33, 1000)])
def test_tree_matches_oracle(fs, oracle, args):
    np.testing.assert_array_equal(fs.build_tree(*args), oracle.build_tree(*args))


def test_tree_rejects_bad_arguments(fs):
    for args in [(0, 1, 1, 5), (10, 0, 1, 5), (10, 1, 0, 5), (10, 1, 1, 0), (1, 1, 1, 5)]:
        with pytest.raises(fs.HodlrError):
            fs.build_tree(*args)


def test_argument_errors_are_reported_before_device_use(fs):
    from fastsolver_b200._lib import lib
    assert lib.hodlr_leaf_solve(-1, 1, None, 1, None, 1, None, None, None) == -1
    assert lib.hodlr_leaf_solve(4, 1, None, 4, None, 4, None, None, None) == -3
    assert lib.hodlr_leaf_solve(4, 1, 8, 3, 8, 4, 8, None, None) == -4
    assert lib.hodlr_gemm_reduce(1.0, 4, 2, 3, 8, 2, 8, 4, 0, 8, 2, None) == -6
    assert lib.hodlr_node_lu_solve(0, 2, 1, 8, 2, 8, 2, 8, 2, 8, 2, None, None) == -1
    assert lib.hodlr_gemm_broadcast(-1.0, 1.0, 4, 2, 2, 8, 4, 0, 8, 2, 1, None) == -11
    assert lib.hodlr_solve(None, None) == -1
    assert lib.hodlr_status_string(-1003) == b"refinement did not reach the tolerance"
    h = ctypes.c_void_p()
    two = (ctypes.c_void_p * 2)(None, None)
    assert lib.hodlr_batch_create(None, two, 2) == -1
    assert lib.hodlr_batch_create(ctypes.byref(h), None, 2) == -2
    assert lib.hodlr_batch_create(ctypes.byref(h), two, 2) == -2   # null system handle
    assert lib.hodlr_batch_create(ctypes.byref(h), two, 0) == -3
    assert h.value is None
    assert lib.hodlr_batch_solve_refined(None, 1e-12, 10, None, None, None, None, None) == -1
    assert lib.hodlr_batch_destroy(None) == -1
    assert lib.hodlr_get_schedule(None, None) == -1
    assert lib.hodlr_set_schedule(None, None) == -1
    assert lib.hodlr_autotune(None, 1, 1e-12, 2, None, None, None, 0, None) == -1
    assert lib.hodlr_batch_autotune(None, 1e-12, 2, None, None, None, 0, None) == -1
    assert lib.hodlr_solve_refined_host(None, None, 0, None, 0, None, 0, None, 0, None, 0, 1,
                                        1e-12, 10, None, None, None) == -1


def test_schedule_cache_key(fs):
    from fastsolver_b200 import autotune
    h = fs.HodlrMatrix(16, 262144, 64, 512)
    assert autotune.shape_key(h, fs.PREC_MIXED) == "N=262144,m=16,r=64,t=512,p=1"
    assert autotune.load("/nonexistent/cache.json") == {}


@pytest.mark.skipif(cuda_available(), reason="checks the no-device status")
def test_no_cpu_fallback_without_device(fs):
    from fastsolver_b200._lib import lib, ERR_CUDA
    h = ctypes.c_void_p()
    assert lib.hodlr_create(ctypes.byref(h), 480, 2, 30, 60) == ERR_CUDA
    assert lib.hodlr_leaf_solve(4, 1, 8, 4, 8, 4, 8, None, None) == ERR_CUDA
