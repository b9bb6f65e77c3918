"""The FP32 GEMM engines against a float64 torch reference.

engine 0 is the FP32 FMA pipe; engine 1 the tcgen05 split-operand tensor-core
kernel (x = hi + lo in BF16, three products hi*hi + hi*lo + lo*hi, FP32
accumulation in tensor memory), whose relative error is bounded by a few
2^-16 of |A||B| -- the tolerance below.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(engine, transa, m, n, k, alpha=1.0, beta=0.0, seed=0):
    import torch
    from fastsolver_b200._lib import lib
    g = torch.Generator(device="cpu").manual_seed(seed)
    Ash = (k, m) if transa else (m, k)
    A = torch.randn(Ash, generator=g, dtype=torch.float32)
    B = torch.randn((k, n), generator=g, dtype=torch.float32)
    C0 = torch.randn((m, n), generator=g, dtype=torch.float32)
    # column-major device copies: transpose of a contiguous (cols, rows) tensor
    Ad = A.t().contiguous().cuda().t()
    Bd = B.t().contiguous().cuda().t()
    Cd = C0.t().contiguous().cuda().t()
    st = lib.hodlr_gemm_f32(transa, m, n, k, alpha, Ad.data_ptr(), Ad.stride(1), Bd.data_ptr(),
                            Bd.stride(1), beta, Cd.data_ptr(), Cd.stride(1), engine, None)
    assert st == 0
    opA = A.double().t() if transa else A.double()
    ref = beta * C0.double() + alpha * (opA @ B.double())
    scale = abs(alpha) * (opA.abs() @ B.double().abs()) + abs(beta) * C0.double().abs()
    err = ((Cd.cpu().double() - ref).abs() / scale.clamp_min(1e-30)).max().item()
    return err


SHAPES = [(128, 128, 32, 0), (448, 592, 64, 0), (64, 592, 64, 0), (512, 528, 64, 0),
          (64, 592, 2048, 1), (64, 80, 4096, 1), (200, 300, 77, 0), (37, 45, 19, 1)]


TC_TOL = 6e-5   # a few 2^-16 of |A||B|


@pytest.mark.parametrize("m,n,k,transa", SHAPES)
def test_tc_split_gemm(fs, cuda, m, n, k, transa):
    err = _run(1, transa, m, n, k, alpha=-1.0, beta=1.0, seed=m + n + k)
    assert err < TC_TOL, err


@pytest.mark.parametrize("alpha,beta", [(0.5, 2.0), (2.0, 0.0), (0.0, 3.0), (-1.5, -0.25)])
def test_tc_split_gemm_scalars(fs, cuda, alpha, beta):
    # the engine folds Cin into the accumulator as (beta / alpha) Cin
    for m, n, k, transa in [(448, 592, 64, 0), (64, 592, 128, 1)]:
        err = _run(1, transa, m, n, k, alpha=alpha, beta=beta, seed=m + k)
        assert err < TC_TOL, (m, n, k, alpha, beta, err)


@pytest.mark.parametrize("m,n,k,transa", SHAPES[:4])
def test_simt_fp32_gemm(fs, cuda, m, n, k, transa):
    err = _run(0, transa, m, n, k, alpha=0.5, beta=2.0, seed=k)
    assert err < 1e-5, err
