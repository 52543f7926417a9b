"""Error paths on the GPU, made to happen without any fault.

- an iterative solve that hits its iteration cap returns status 1 (a usable
  result with a warning) and reports the iteration count, as the reference
  reports its KSP iterations and true residual (SolveFem.cpp:142-152);
- a non-finite density is rejected with TOPO_ERR_NAN and the context stays
  usable;
- the bounded device waits (the MMA dual solve's grid barrier, the block
  operator's bulk-copy waits) are made to run out by a barrier that never
  opens / a copy that is never issued (topo_test_wait_limits hold=1): the
  call returns TOPO_ERR_TIMEOUT, and the next call on the same context gives
  the oracle's result;
- a serving job is cancelled while queued and while running (between two
  design iterations); the other jobs finish unchanged.
"""
import threading
import time

import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

KW = dict(Emax=1.0, rmin=1.5, volfrac=0.12)


def dev(cuda, a):
    return cuda.tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")


@pytest.fixture(scope="module")
def mesh(T):
    return T.gen_cantilever(16, 8, 6, 8)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_fgmres_iteration_cap_returns_status_1(T, cuda, mesh, prec):
    v, e, f, ld, lv = mesh
    pr = T.PREC_MIXED if prec == "mixed" else T.PREC_FP64
    ctx = T.Context(v, e, f, ld, lv, precision=pr, fem_maxit=2, fem_rtol=1e-10, **KW)
    x = dev(cuda, np.full(e.shape[0], 0.3))
    fx, gx, df, dg, rc = ctx.fem_obj_sens(x)
    info = ctx.info()
    assert rc == T.TOPO_NOT_CONVERGED
    assert info.fem_status == 1 and info.fem_its == 2
    assert np.isfinite(fx) and info.fem_relres > 1e-10
    # the same context converges once the cap allows it
    ctx.set_params(fem_maxit=10000)
    fx2, _, _, _, rc2 = ctx.fem_obj_sens(x)
    assert rc2 == 0 and ctx.info().fem_status == 0 and ctx.info().fem_its > 2
    ctx.close()


def test_filter_cg_iteration_cap_returns_status_1(T, cuda, mesh):
    v, e, f, ld, lv = mesh
    ctx = T.Context(v, e, f, ld, lv, filter_maxit=1, filter_rtol=1e-14, **KW)
    x = dev(cuda, np.random.default_rng(3).uniform(0, 1, e.shape[0]))
    rc = T.lib().topo_filter_apply(ctx.h, T._dptr(x), T._dptr(ctx.zeros(ctx.ne)), 0.01)
    assert rc == T.TOPO_NOT_CONVERGED and ctx.info().filter_its[0] == 1
    ctx.close()


def test_nan_density_rejected_and_context_recovers(T, O, cuda, mesh):
    v, e, f, ld, lv = mesh
    tight = dict(fem_rtol=1e-10, filter_rtol=1e-12)
    ctx = T.Context(v, e, f, ld, lv, **KW, **tight)
    x = np.random.default_rng(4).uniform(0.05, 1.0, e.shape[0])
    bad = x.copy()
    bad[e.shape[0] // 3] = np.nan
    with pytest.raises(T.TopoError) as ei:
        ctx.fem_obj_sens(dev(cuda, bad))
    assert ei.value.code == T.TOPO_ERR_NAN
    fx, gx, df, dg, rc = ctx.fem_obj_sens(dev(cuda, x))
    orc = O.Oracle(v, e, f, ld, lv, **KW, **tight)
    ofx, ogx, odf, odg = orc.fem_obj_sens(x)
    assert rc == 0 and abs(fx - ofx) <= 1e-8 * abs(ofx)
    assert rel(df.cpu().numpy(), odf) < 1e-7
    ctx.close()
    orc.close()


def test_mma_grid_barrier_timeout(T, O, cuda, mesh):
    """The dual solve's grid barrier never opens (hold): every block's wait
    runs out after a short spin limit, the call returns TOPO_ERR_TIMEOUT, and
    the next update on the same context matches the oracle."""
    v, e, f, ld, lv = mesh
    ctx = T.Context(v, e, f, ld, lv, **KW)
    orc = O.Oracle(v, e, f, ld, lv, **KW)
    n = e.shape[0]
    rng = np.random.default_rng(12)
    x1 = rng.uniform(0.05, 0.6, n)
    df1, dg1 = -rng.uniform(0.1, 3.0, n), rng.uniform(0.5, 1.5, n) / n
    gx1 = np.array([x1.mean() - 0.3])
    ctx.test_wait_limits(barrier_spins=1 << 12, hold=1)
    mn, mx = ctx.mma_movelimit(dev(cuda, x1))
    with pytest.raises(T.TopoError) as ei:
        ctx.mma_update(dev(cuda, x1), dev(cuda, df1), gx1, dev(cuda, dg1), mn, mx)
    assert ei.value.code == T.TOPO_ERR_TIMEOUT
    omn, omx = orc.mma_movelimit(x1)
    orc.mma_update(x1, df1, gx1, dg1, omn, omx)  # the oracle's first update completes
    # normal operation again: the second update agrees with the oracle's
    # (GenSub's first two iterations do not use the failed update's x)
    ctx.test_wait_limits()
    x2 = rng.uniform(0.05, 0.6, n)
    df2, dg2 = -rng.uniform(0.1, 3.0, n), rng.uniform(0.5, 1.5, n) / n
    gx2 = np.array([x2.mean() - 0.3])
    mn, mx = ctx.mma_movelimit(dev(cuda, x2))
    xn = ctx.mma_update(dev(cuda, x2), dev(cuda, df2), gx2, dev(cuda, dg2), mn, mx).cpu().numpy()
    omn, omx = orc.mma_movelimit(x2)
    oxn = orc.mma_update(x2, df2, gx2, dg2, omn, omx)
    assert rel(xn, oxn) < 1e-8
    assert ctx.info().mma_inner_its > 0
    ctx.close()
    orc.close()


def test_block_operator_copy_timeout(T, O, cuda):
    """The block operator's waits for its bulk copies of element matrices run
    out when no copy is issued (hold): TOPO_ERR_TIMEOUT, and the next
    application on the same context equals the per-case oracle."""
    v, e, f, _, _ = T.gen_cantilever(10, 5, 4, 8)
    ld, lv = T.gen_multiload(10, 5, 4, 3)
    cp = np.arange(0, 10, 3, dtype=np.int32)
    ctx = T.Context(v, e, f, ld, lv, case_ptr=cp, **KW)
    rng = np.random.default_rng(13)
    x = rng.uniform(0.01, 1.0, e.shape[0])
    u = rng.standard_normal(3 * 3 * v.shape[0])
    ctx.test_wait_limits(copy_cycles=1 << 20, hold=1)
    with pytest.raises(T.TopoError) as ei:
        ctx.fem_apply_block(dev(cuda, x), dev(cuda, u))
    assert ei.value.code == T.TOPO_ERR_TIMEOUT
    ctx.test_wait_limits()
    y = ctx.fem_apply_block(dev(cuda, x), dev(cuda, u)).cpu().numpy()
    orc = O.Oracle(v, e, f, ld, lv, case_ptr=cp, **KW)
    orc.assemble(x)
    n = 3 * v.shape[0]
    for k in range(3):
        assert rel(y[k * n:(k + 1) * n], orc.kmatvec(u[k * n:(k + 1) * n])) < 1e-12
    ctx.close()
    orc.close()


def test_server_job_cancelled_queued_and_running(T, cuda):
    v, e, f, ld, lv = T.gen_cantilever(12, 6, 4, 8)
    kw = dict(KW, fem_rtol=1e-5, ch_tol=0.0)
    s = T.Server(hbm_budget_bytes=0, max_active=4)
    a = s.submit(v, e, f, ld, lv, iterations=6, **kw)
    b = s.submit(v, e, f, ld, lv, iterations=5000, **kw)  # cancelled while running
    c = s.submit(v, e, f, ld, lv, iterations=6, arrival_s=30.0, **kw)  # cancelled while queued
    s.cancel(c)
    t = threading.Thread(target=lambda: (time.sleep(1.5), s.cancel(b)))
    t.start()
    t0 = time.perf_counter()
    s.run()
    t.join()
    assert time.perf_counter() - t0 < 25.0  # c's arrival at 30 s is never waited for
    ja, jb, jc = s.job(a), s.job(b), s.job(c)
    assert ja["rc"] == 0 and len(ja["fx"]) == 6
    assert jb["rc"] == T.TOPO_ERR_CANCELLED and 1 <= len(jb["fx"]) < 5000
    assert jc["rc"] == T.TOPO_ERR_CANCELLED and len(jc["fx"]) == 0
    # the iterations b finished are the same as a's (same job, same start)
    k = min(len(jb["fx"]), 6)
    assert rel(jb["fx"][:k], ja["fx"][:k]) < 1e-6
    st = s.stats()
    assert st["jobs_done"] == 1 and st["jobs_failed"] == 0
    s.close()
