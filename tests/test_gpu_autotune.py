"""Launch schedules and the autotuner.

Every schedule computes the same solve: each one must reach the same
accuracy against the oracle (FP64 fused to 1e-12; mixed refined to relres
<= 1e-12).  The autotuner must return a valid schedule that was measured,
install it, and leave the system solvable.
"""
import numpy as np
import pytest

from gpu_util import relerr

pytestmark = pytest.mark.gpu

N, M, R, T = 20000, 4, 24, 512


@pytest.fixture(scope="module")
def system(oracle):
    return oracle.gaussian_system(N, M, R, T, seed=77)


def _load(fs, s, n=N, m=M, r=R, t=T):
    h = fs.HodlrMatrix(m, n, r, t).create_tree()
    h.set_matrix(s.D, s.U, s.V)
    h.set_rhs(s.B)
    return h


@pytest.mark.parametrize("sched", [
    dict(leaf_ob32=0), dict(leaf_ob32=256), dict(leaf_nb=32), dict(leaf_nb=32, leaf_ob32=64),
    dict(reduce_rows=256, bcast_rows=2048), dict(reduce_rows=4096, bcast_rows=16)])
def test_mixed_schedules_same_accuracy(fs, oracle, cuda, system, sched):
    h = _load(fs, system)
    h.schedule = sched
    assert {k: h.schedule[k] for k in sched} == sched
    it, rr = fs.FastSolver().solve_refined(h, fs.PREC_MIXED, tol=1e-12, maxiter=10)
    assert rr <= 1e-12
    Xo, _ = oracle.bfs_solve(system, nthreads=8)
    assert relerr(h.solution(), Xo[:, :M]) < 1e-11


@pytest.mark.parametrize("ob64", [64, 128, 256])
def test_fp64_two_level_leaf_matches_oracle(fs, oracle, cuda, system, ob64):
    h = _load(fs, system)
    h.schedule = dict(leaf_ob64=ob64, reduce_rows=1024)
    fs.FastSolver().bfs_solve(h)
    Xo, _ = oracle.bfs_solve(system, nthreads=8)
    assert relerr(h.solution(), Xo[:, :M]) < 1e-12


def test_fp64_two_level_leaf_large_grid(fs, oracle, cuda):
    """The block-row solves of the two-level FP64 leaf LU are in-place products
    (C = L^{-1} C): with 256 leaves their launches hold thousands of tiles,
    and a tiling that split one item's 128 rows over two CTAs would let one
    CTA overwrite rows the other still reads."""
    s = oracle.gaussian_system(131072, 4, 32, 512, seed=41)
    h = _load(fs, s, 131072, 4, 32, 512)
    h.schedule = dict(leaf_ob64=128)
    fs.FastSolver().bfs_solve(h)
    Xo, _ = oracle.bfs_solve(s, nthreads=8)
    assert relerr(h.solution(), Xo[:, :4]) < 1e-12


def test_fp64_two_level_leaf_1024_rows(fs, oracle, cuda):
    """Leaves above 512 rows take 16-wide FP64 panels: 8 of them per block."""
    s = oracle.gaussian_system(9001, 3, 40, 1024, seed=5)
    h = _load(fs, s, 9001, 3, 40, 1024)
    h.schedule = dict(leaf_ob64=128)
    fs.FastSolver().bfs_solve(h)
    Xo, _ = oracle.bfs_solve(s, nthreads=8)
    assert relerr(h.solution(), Xo[:, :3]) < 1e-12


def test_invalid_schedules_rejected(fs, cuda, system):
    h = fs.HodlrMatrix(2, 9001, 20, 1024).create_tree()   # leaves above 512 rows
    with pytest.raises(fs.HodlrError):
        h.schedule = dict(leaf_nb=64)
    h2 = _load(fs, system)
    for bad in (dict(reduce_rows=17), dict(bcast_rows=0), dict(leaf_ob32=-1), dict(leaf_nb=48)):
        with pytest.raises(fs.HodlrError):
            h2.schedule = bad


def test_new_schedule_needs_new_factors(fs, cuda, system):
    h = _load(fs, system)
    sol = fs.FastSolver()
    sol.factor(h, fs.PREC_MIXED)
    h.schedule = dict(bcast_rows=1024)
    with pytest.raises(fs.HodlrError) as e:
        sol.solve(h)
    assert e.value.status == fs.ERR_STATE


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_autotune_installs_a_measured_schedule(fs, oracle, cuda, system, precision):
    prec = fs.PREC_MIXED if precision == "mixed" else fs.PREC_FP64
    h = _load(fs, system)
    best, ms, trials = h.autotune(prec, tol=1e-12, reps=1)
    assert ms > 0 and len(trials) >= 5
    assert best == h.schedule
    assert any(t[0] == best and t[1] == ms for t in trials)
    h.set_rhs(system.B)
    if prec == fs.PREC_MIXED:
        it, rr = fs.FastSolver().solve_refined(h, prec, tol=1e-12)
        assert rr <= 1e-12
    else:
        fs.FastSolver().bfs_solve(h)
    Xo, _ = oracle.bfs_solve(system, nthreads=8)
    assert relerr(h.solution(), Xo[:, :M]) < 1e-11


def test_batch_autotune(fs, oracle, cuda):
    cfgs = [(8192, 2, 16, 256), (12000, 20, 40, 512), (6000, 5, 30, 400)]
    pairs = []
    for i, (n, m, r, t) in enumerate(cfgs):
        s = oracle.gaussian_system(n, m, r, t, seed=900 + i)
        pairs.append((s, _load(fs, s, n, m, r, t)))
    batch = fs.SystemBatch([h for _, h in pairs])
    best, ms, trials = batch.autotune(tol=1e-12, reps=1)
    assert ms > 0 and len(trials) >= 5
    for _, h in pairs:
        assert h.schedule == best
    for s, h in pairs:
        h.set_rhs(s.B)
    it, rr = batch.solve_refined(tol=1e-12)
    for (s, h), (n, m, r, t), x in zip(pairs, cfgs, rr):
        assert x <= 1e-12
        Xo, _ = oracle.bfs_solve(s, nthreads=8)
        assert relerr(h.solution(), Xo[:, :m]) < 1e-11
