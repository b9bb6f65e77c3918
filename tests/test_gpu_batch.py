"""Batched solve of independent uneven systems against the oracle.

Systems of different size, rank, leaf size and right-hand-side count are
merged into one schedule (SystemBatch); each system's solution must match the
oracle's FP64 walk of that system alone, with relative residual <= 1e-12,
exactly as when the system is solved by itself.
"""
import numpy as np
import pytest

from gpu_util import relerr

pytestmark = pytest.mark.gpu

# (N, nrhs, rank, threshold): uneven in every parameter, as the batched
# workload draws them (N log-uniform, leaf in {256, 512, 1024}, rank 16..96,
# 1..32 right-hand sides), at sizes the oracle finishes in seconds
SYSTEMS = [(8192, 1, 16, 256), (12000, 7, 40, 512), (9001, 32, 24, 1024),
           (20000, 3, 96, 512), (4096, 16, 64, 256), (16384, 2, 50, 1024)]


def _load(fs, oracle, N, m, r, t, seed):
    s = oracle.gaussian_system(N, m, r, t, seed=seed)
    h = fs.HodlrMatrix(m, N, r, t).create_tree()
    h.set_matrix(s.D, s.U if s.U.shape[1] else None, s.V if s.V.shape[1] else None)
    h.set_rhs(s.B)
    return s, h


def _check(oracle, s, h, m, rr, stream=None):
    assert rr <= 1e-12
    x = h.solution(stream=stream)
    assert oracle.relres(s, x) <= 2e-12
    Xo, _ = oracle.bfs_solve(s, nthreads=8)
    assert relerr(x, Xo[:, :m]) < 1e-11


def test_batch_uneven_vs_oracle(fs, oracle, cuda):
    pairs = [_load(fs, oracle, *cfg, seed=100 + i) for i, cfg in enumerate(SYSTEMS)]
    batch = fs.SystemBatch([h for _, h in pairs])
    fs.reset_launch_count()
    it, rr = batch.solve_refined(tol=1e-12, maxiter=10)
    launches = fs.launch_count()
    assert 1 <= it <= 4
    for (s, h), cfg, r in zip(pairs, SYSTEMS, rr):
        _check(oracle, s, h, cfg[1], r)
    # merged schedules: fewer launches than the systems solved one by one
    fs.reset_launch_count()
    for s, h in pairs:
        h.set_rhs(s.B)
        fs.FastSolver().solve_refined(h, fs.PREC_MIXED, tol=1e-12, maxiter=it)
    assert launches < fs.launch_count()


def test_batch_launches_do_not_grow_with_systems(fs, oracle, cuda):
    """Systems of one kernel class (same leaf panel width, <= 16 RHS) share
    every launch: a batch of five costs the launches of its deepest member
    plus the per-level steps the others add, not five solves."""
    cfgs = [(8192, 4, 16, 512), (12000, 1, 40, 512), (20000, 16, 30, 400),
            (6000, 8, 24, 512), (16384, 2, 50, 300)]
    pairs = [_load(fs, oracle, *cfg, seed=500 + i) for i, cfg in enumerate(cfgs)]
    single = []
    for s, h in pairs:
        fs.reset_launch_count()
        it1, _ = fs.FastSolver().solve_refined(h, fs.PREC_MIXED, tol=0.0, maxiter=2,
                                               check_conv=False)
        single.append(fs.launch_count())
    batch = fs.SystemBatch([h for _, h in pairs])
    for s, h in pairs:
        h.set_rhs(s.B)
    fs.reset_launch_count()
    it, rr = batch.solve_refined(tol=0.0, maxiter=2, check_conv=False)
    assert it == 2
    assert fs.launch_count() <= 1.2 * max(single)
    for (s, h), cfg, r in zip(pairs, cfgs, rr):
        _check(oracle, s, h, cfg[1], r)


def test_batch_graph_replay_new_rhs(fs, oracle, cuda):
    """On a side stream the factor pass and the sweep are captured as CUDA
    graphs on first use; new right-hand sides loaded into the same systems
    are then solved by replay, as accurately as the first."""
    import torch
    cfgs = SYSTEMS[:4]
    pairs = [_load(fs, oracle, *cfg, seed=200 + i) for i, cfg in enumerate(cfgs)]
    batch = fs.SystemBatch([h for _, h in pairs])
    st = torch.cuda.Stream()
    rng = np.random.default_rng(7)
    for trial in range(3):
        for (s, h), cfg in zip(pairs, cfgs):
            s.B = np.asfortranarray(rng.standard_normal((cfg[0], cfg[1])))
            h.set_rhs(s.B, stream=st)
        it, rr = batch.solve_refined(tol=1e-12, maxiter=10, stream=st)
        st.synchronize()
        for (s, h), cfg, r in zip(pairs, cfgs, rr):
            _check(oracle, s, h, cfg[1], r, stream=st)


@pytest.mark.parametrize("order", ["large_leaves_first", "small_leaves_first"])
def test_batch_graph_replay_leaf_groups_both_orders(fs, oracle, cuda, order):
    """Two leaf groups of the 17..32-column apply class (leaves up to 1024
    rows and up to 512 rows, different dynamic shared memory) captured in
    one graph, built in either order, then replayed with new right-hand
    sides: the kernel's shared-memory limit only ever rises, so every
    captured node can launch on replay."""
    import torch
    cfgs = [(9001, 32, 24, 1024), (12000, 32, 40, 512)]
    if order == "small_leaves_first":
        cfgs = cfgs[::-1]
    pairs = [_load(fs, oracle, *cfg, seed=300 + i) for i, cfg in enumerate(cfgs)]
    batch = fs.SystemBatch([h for _, h in pairs])
    st = torch.cuda.Stream()
    rng = np.random.default_rng(11)
    for trial in range(3):
        for (s, h), cfg in zip(pairs, cfgs):
            s.B = np.asfortranarray(rng.standard_normal((cfg[0], cfg[1])))
            h.set_rhs(s.B, stream=st)
        it, rr = batch.solve_refined(tol=1e-12, maxiter=10, stream=st)
        st.synchronize()
        for (s, h), cfg, r in zip(pairs, cfgs, rr):
            _check(oracle, s, h, cfg[1], r, stream=st)
    batch.close()


def test_batch_leaves_systems_factored(fs, oracle, cuda):
    """After a batch solve every system holds its mixed factors: a plain
    hodlr_solve of a new RHS applies them (FP32 accuracy, no refinement)."""
    pairs = [_load(fs, oracle, *cfg, seed=300 + i) for i, cfg in enumerate(SYSTEMS[:3])]
    fs.SystemBatch([h for _, h in pairs]).solve_refined()
    s, h = pairs[1]
    B2 = np.asfortranarray(np.random.default_rng(3).standard_normal(s.B.shape))
    h.set_rhs(B2)
    fs.FastSolver().solve(h)
    s.B = B2
    Xo, _ = oracle.bfs_solve(s, nthreads=8)
    assert relerr(h.solution(), Xo[:, :s.B.shape[1]]) < 1e-4


def test_batch_reports_failing_system(fs, oracle, cuda):
    pairs = [_load(fs, oracle, *cfg, seed=400 + i) for i, cfg in enumerate(SYSTEMS[:3])]
    s, h = pairs[2]
    s.D[300, :] = 0.0      # zero row in a leaf of system 2 -> exact zero pivot
    h.set_matrix(s.D, s.U, s.V)
    batch = fs.SystemBatch([h for _, h in pairs])
    with pytest.raises(fs.HodlrError) as e:
        batch.solve_refined()
    assert e.value.status > 0
    assert batch.failed == 2


def test_batch_of_one_matches_single_solve(fs, oracle, cuda):
    s, h = _load(fs, oracle, 20000, 4, 24, 512, seed=5)
    it, rr = fs.SystemBatch([h]).solve_refined()
    x_batch = h.solution()
    h.set_rhs(s.B)
    it1, rr1 = fs.FastSolver().solve_refined(h, fs.PREC_MIXED)
    assert it == it1
    np.testing.assert_allclose(rr[0], rr1, rtol=1e-6)
    assert relerr(x_batch, h.solution()) < 1e-14
