"""The device-driven design iteration (step_graph = 1) and the batch of
independent design instances (topo_opt_step_batch).

From the second iteration of a run on, the whole main.cpp:72-112 loop body is
replayed from CUDA graphs in which the FGMRES restart cycles, the Arnoldi
steps and the filter CG iterations are conditional nodes decided on the
device.  The same kernels run in the same order as in a host-driven step, so
the trajectories agree to rounding: bar 1e-6 relative compliance per
iteration (the element scatter's float atomics make two runs differ in the
last bits, which an FGMRES stopping test can turn into one more or one fewer
iteration), volume constraint 1e-9.  A batch advances several instances of
different sizes and options at once; each instance's trajectory must equal
its own solo run by the same bar.
"""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

KW = dict(Emax=1.0, rmin=1.5, volfrac=0.12, fem_rtol=1e-5, ch_tol=0.0)


def run(T, mesh, n, **kw):
    ctx = T.Context(*mesh, stream="own", **dict(KW, **kw))
    ctx.opt_init()
    h = ctx.opt_run(n)
    its = ctx.info().fem_its
    assert ctx.info().step_graph == kw.get("step_graph", 0)  # replayed (1) or direct (0) as asked
    xp = ctx.opt_tensor(1).cpu().numpy()
    ctx.close()
    return h, xp, its


@pytest.mark.parametrize("prec,nen,tune", [("fp64", 8, 1), ("mixed", 8, 1), ("mixed", 4, 1), ("mixed", 8, 0)])
def test_graph_step_matches_direct_step(T, cuda, prec, nen, tune):
    mesh = T.gen_cantilever(40, 20, 10, 8) if nen == 8 else T.gen_cantilever(12, 6, 6, 4)
    pr = T.PREC_MIXED if prec == "mixed" else T.PREC_FP64
    hd, xd, _ = run(T, mesh, 12, precision=pr, step_graph=0, autotune=tune)
    hg, xg, its = run(T, mesh, 12, precision=pr, step_graph=1, autotune=tune)
    assert its > 0
    assert rel(hg[:, 0], hd[:, 0]) < 1e-6
    assert np.abs(hg[:, 1] - hd[:, 1]).max() < 1e-9
    assert np.abs(hg[:, 2] - hd[:, 2]).max() < 1e-6
    assert np.abs(xg - xd).max() < 1e-5


def test_graph_step_with_projection_crosses_beta_steps(T, cuda):
    """proj = 1 through iteration 32: beta moves at iteration 30 on the device
    (PDEFilter.cpp:260-268) exactly as on the host."""
    mesh = T.gen_cantilever(16, 8, 6, 8)
    hd, xd, _ = run(T, mesh, 32, proj=1, step_graph=0)
    hg, xg, _ = run(T, mesh, 32, proj=1, step_graph=1)
    assert rel(hg[:, 0], hd[:, 0]) < 1e-6
    assert np.abs(xg - xd).max() < 1e-5


def test_graph_step_info_and_launch_count(T, cuda):
    mesh = T.gen_cantilever(24, 12, 8, 8)
    ctx = T.Context(*mesh, stream="own", step_graph=1, **KW)
    ctx.opt_init()
    ctx.opt_step()                      # direct: allocates, tunes
    assert ctx.info().step_graph == 0
    l0 = T.kernel_launches()
    it, fx, gx, ch = ctx.opt_step()     # captured, then replayed
    l1 = T.kernel_launches()
    inf = ctx.info()
    assert it == 2 and np.isfinite(fx) and ch > 0
    assert inf.fem_its > 0 and inf.fem_status == 0 and 0 < inf.fem_relres < 1e-5
    assert inf.filter_its[0] > 0 and inf.filter_its[1] > 0 and inf.mma_inner_its > 0
    assert inf.step_graph == 1
    assert l1 - l0 > 100                # the replay counts the kernels it ran
    ctx.close()


def test_graph_step_iteration_cap_and_nan(T, cuda):
    mesh = T.gen_cantilever(16, 8, 6, 8)
    ctx = T.Context(*mesh, stream="own", step_graph=1, **KW)
    ctx.opt_init()
    ctx.opt_step()
    ctx.set_params(fem_maxit=3)         # a new graph with the new cap
    rc = T.lib().topo_opt_step(ctx.h, None, None, None, None)
    assert rc == T.TOPO_NOT_CONVERGED and ctx.info().fem_its == 3 and ctx.info().fem_status == 1
    assert ctx.info().step_graph == 1
    ctx.set_params(fem_maxit=10000)
    # a non-finite density inside the device-resident design is reported
    xp = T.device_view(ctx.opt_vector(1), ctx.ne)
    xp[5] = float("nan")
    with pytest.raises(T.TopoError) as ei:
        ctx.opt_step()
    assert ei.value.code == T.TOPO_ERR_NAN
    ctx.opt_init()                      # a fresh run works again
    h = ctx.opt_run(4)
    assert np.all(np.isfinite(h)) and h.shape == (4, 3)
    ctx.close()


def test_batch_of_instances_equals_solo_runs(T, cuda):
    """Four independent design instances (hex8 and tet4, different sizes,
    volume fractions and filter radii, FP64 and mixed) advanced together by
    topo_opt_step_batch for 10 iterations: each trajectory equals the
    instance's solo host-driven run."""
    specs = [((24, 12, 8, 8), dict(volfrac=0.12, rmin=1.5, precision=1)),
             ((16, 8, 8, 4), dict(volfrac=0.2, rmin=1.3, precision=1)),
             ((30, 15, 10, 8), dict(volfrac=0.25, rmin=1.8, precision=0)),
             ((12, 6, 4, 8), dict(volfrac=0.15, rmin=2.0, precision=1))]
    n = 10
    solo = []
    for dims, kw in specs:
        h, _, _ = run(T, T.gen_cantilever(*dims), n, step_graph=0, **kw)
        solo.append(h[:, 0])
    ctxs = []
    for dims, kw in specs:
        c = T.Context(*T.gen_cantilever(*dims), stream="own", step_graph=1, **dict(KW, **kw))
        c.opt_init()
        ctxs.append(c)
    hist = np.zeros((n, len(ctxs)))
    caps = []
    for it in range(n):
        st, fx = T.opt_step_batch(ctxs)
        assert np.all(st == 0), st
        hist[it] = fx
        caps.append(ctxs[0].info().t_capture_ms)
    for k in range(len(ctxs)):
        assert rel(hist[:, k], solo[k]) < 1e-6, k
        # replayed as a branch of the one batch graph
        assert ctxs[k].info().fem_its > 0 and ctxs[k].info().step_graph == 2
    # the batch graph is captured once (second call) and then reused
    assert caps[1] > 0 and all(c == caps[1] for c in caps[2:])
    for c in ctxs:
        c.close()


def test_batch_graph_follows_set_and_options(T, cuda):
    """The batch graph is keyed by the ordered set of instances and by their
    own captures: a smaller set, an instance with new options (an iteration
    cap) and a destroyed instance each lead to a graph of their own, and the
    trajectories still equal the solo runs."""
    specs = [((20, 10, 6, 8), dict(volfrac=0.12)), ((12, 6, 6, 4), dict(volfrac=0.2, rmin=1.3)),
             ((16, 8, 8, 8), dict(volfrac=0.25, precision=1))]
    n = 9
    solo = [run(T, T.gen_cantilever(*d), n, step_graph=0, **kw)[0][:, 0] for d, kw in specs]
    ctxs = [T.Context(*T.gen_cantilever(*d), stream="own", step_graph=1, **dict(KW, **kw)) for d, kw in specs]
    for c in ctxs:
        c.opt_init()
    hist = [[] for _ in ctxs]

    def step(ks):
        st, fx = T.opt_step_batch([ctxs[k] for k in ks])
        for j, k in enumerate(ks):
            hist[k].append(fx[j])
        return st

    for _ in range(3):
        assert np.all(step([0, 1, 2]) == 0)
    for _ in range(2):                      # a subset, in another order
        assert np.all(step([2, 0]) == 0)
    assert ctxs[0].info().step_graph == 2
    step([1])                               # alone: its own graphs
    step([1])
    assert ctxs[1].info().step_graph == 1
    # an iteration cap on one instance: its graphs and the batch graph are
    # captured again; the cap shows in its status only
    ctxs[2].set_params(fem_maxit=2)
    st = step([0, 1, 2])
    assert st[2] == T.TOPO_NOT_CONVERGED and st[0] == 0 and st[1] == 0
    assert ctxs[2].info().fem_its == 2 and ctxs[2].info().step_graph == 2
    ctxs[2].close()                         # destroyed: batch graphs naming it go
    for _ in range(2):
        assert np.all(step([0, 1]) == 0)
    assert len(hist[0]) == n - 1 and len(hist[1]) == n - 1
    for k in (0, 1):
        assert rel(np.array(hist[k]), solo[k][: n - 1]) < 1e-6, k
    assert rel(np.array(hist[2][:5]), solo[2][:5]) < 1e-6
    for c in ctxs[:2]:
        c.close()


def test_async_steps_from_one_thread_equal_solo_runs(T, cuda):
    """topo_opt_step_async / topo_opt_step_query: three instances kept going
    from one host thread, each relaunched as soon as its iteration is done,
    equal their solo host-driven runs; a context with an iteration in flight
    refuses other optimisation calls."""
    specs = [((20, 10, 6, 8), dict(volfrac=0.12)), ((12, 6, 6, 4), dict(volfrac=0.2, rmin=1.3)),
             ((16, 8, 8, 8), dict(volfrac=0.25, precision=1))]
    n = 8
    solo = [run(T, T.gen_cantilever(*d), n, step_graph=0, **kw)[0][:, 0] for d, kw in specs]
    ctxs = [T.Context(*T.gen_cantilever(*d), stream="own", step_graph=1, **dict(KW, **kw)) for d, kw in specs]
    for c in ctxs:
        c.opt_init()
    hist = [[] for _ in ctxs]
    running = [False] * len(ctxs)
    checked = False
    while min(len(h) for h in hist) < n:
        for k, c in enumerate(ctxs):
            if len(hist[k]) >= n:
                continue
            if not running[k]:
                c.opt_step_async()
                running[k] = True
                if len(hist[k]) >= 2 and not checked:  # a replayed iteration is in flight
                    with pytest.raises(T.TopoError):
                        c.opt_step()
                    checked = True
                continue
            r = c.opt_step_query()
            if r is not None:
                rc, it, fx, gx, ch = r
                assert rc == 0 and it == len(hist[k]) + 1
                hist[k].append(fx)
                running[k] = False
    assert checked
    for k, c in enumerate(ctxs):
        assert rel(np.array(hist[k]), solo[k]) < 1e-6, k
        assert c.info().step_graph == 1
        c.close()
