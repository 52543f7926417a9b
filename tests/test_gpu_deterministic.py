"""Bitwise-reproducible runs (deterministic = 1).

The default element operators add each element's contributions into the
node vectors with atomics, so two runs of the same job agree only to
rounding.  With deterministic = 1 every node sums its elements'
contributions in the fixed order of the node-to-element map, no launch shape
is timed, and several load cases are solved one by one.  Two runs of the same
job on the same GPU then give the same bits: every design iteration's
compliance, volume constraint and design change, and the final design.
Against the atomic form the results agree to rounding (the operator to
1e-12, the trajectory at the loop tests' 1e-6 replay bar)."""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

KW = dict(Emax=1.0, rmin=1.5, volfrac=0.12, fem_rtol=1e-5, ch_tol=0.0)


def _run(T, mesh, n, **kw):
    v, e, f, ld, lv = mesh
    ctx = T.Context(v, e, f, ld, lv, **{**KW, **kw})
    ctx.opt_init()
    hist = ctx.opt_run(n)
    x = ctx.opt_tensor(0).cpu().numpy().copy()
    xp = ctx.opt_tensor(1).cpu().numpy().copy()
    its = ctx.info().fem_its
    ctx.close()
    return hist, x, xp, its


@pytest.mark.parametrize("nen,dims", [(8, (24, 12, 8)), (4, (10, 6, 4))])
@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("graphs", [0, 1])
def test_two_runs_give_the_same_bits(T, cuda, nen, dims, prec, graphs):
    """Two fresh contexts of the same job: identical per-iteration compliance,
    constraint and design change, identical final design (==, not a tolerance),
    with host-driven steps and with steps replayed from the step graphs."""
    mesh = T.gen_cantilever(*dims, nen)
    kw = dict(precision=T.PREC_FP64 if prec == 0 else T.PREC_MIXED, deterministic=1, step_graph=graphs)
    a = _run(T, mesh, 8, **kw)
    b = _run(T, mesh, 8, **kw)
    assert np.array_equal(a[0], b[0]), np.abs(a[0] - b[0]).max()
    assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])
    assert a[3] == b[3]
    # the atomic form follows the same trajectory to rounding
    c = _run(T, mesh, 8, precision=kw["precision"], step_graph=graphs)
    assert np.abs(a[0][:, 0] - c[0][:, 0]).max() <= 1e-6 * np.abs(c[0][:, 0]).max()


def test_operators_match_the_atomic_form(T, cuda):
    """K(x) u through the fixed-order gather equals the atomic scatter to
    rounding, and repeated applications give the same bits."""
    import torch
    v, e, f, ld, lv = T.gen_cantilever(20, 10, 6, 8)
    rng = np.random.default_rng(5)
    x = torch.tensor(rng.uniform(0.05, 1.0, e.shape[0]), device="cuda")
    u = torch.tensor(rng.standard_normal(3 * v.shape[0]), device="cuda")
    det = T.Context(v, e, f, ld, lv, deterministic=1, **KW)
    ato = T.Context(v, e, f, ld, lv, **KW)
    y1 = det.fem_apply(x, u).cpu().numpy()
    y2 = det.fem_apply(x, u).cpu().numpy()
    y0 = ato.fem_apply(x, u).cpu().numpy()
    assert np.array_equal(y1, y2)
    assert rel(y1, y0) < 1e-12
    f1 = det.filter(x)
    f2 = det.filter(x)
    f0 = ato.filter(x)
    assert torch.equal(f1, f2)
    assert rel(f1.cpu().numpy(), f0.cpu().numpy()) < 1e-9
    det.close()
    ato.close()


def test_load_cases_one_by_one_reproducible(T, cuda):
    """Several load cases: the deterministic form solves them one by one, with
    the same bits in two runs, and matches the block solve to rounding."""
    import torch
    nx, ny, nz, k = 16, 8, 6, 3
    v, e, f, _, _ = T.gen_cantilever(nx, ny, nz, 8)
    ld, lv = T.gen_multiload(nx, ny, nz, k, 3)
    cp = np.arange(0, 3 * k + 1, 3, dtype=np.int32)
    x = torch.tensor(np.random.default_rng(2).uniform(0.1, 1.0, e.shape[0]), device="cuda")
    out = []
    for det in (1, 1, 0):
        ctx = T.Context(v, e, f, ld, lv, case_ptr=cp, deterministic=det, **{**KW, "fem_rtol": 1e-8})
        fx, gx, df, dg, rc = ctx.fem_obj_sens(x)
        assert rc == 0
        out.append((fx, df.cpu().numpy()))
        ctx.close()
    assert out[0][0] == out[1][0] and np.array_equal(out[0][1], out[1][1])
    assert abs(out[0][0] - out[2][0]) <= 1e-7 * abs(out[2][0])
