"""Parity of every stage of the design iteration, GPU (through the C ABI)
against the CPU oracle on the same seeded inputs.

Tolerances (FP64): element matrices, volumes, K u: 1e-12 relative (summation
order only); tightly converged solves (rtol 1e-10 / 1e-12 on both sides):
compliance 1e-8 and displacements 1e-7 relative (the parity bar of the FP64 solve);
filter 1e-9; MMA update 1e-8; design change exact to 1e-12."""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

KW = dict(Emax=1.0, rmin=1.5, volfrac=0.12)
TIGHT = dict(fem_rtol=1e-10, filter_rtol=1e-12)


@pytest.fixture(scope="module", params=[8, 4], ids=["hex8", "tet4"])
def pair(request, T, O, cuda):
    nen = request.param
    dims = (16, 8, 6) if nen == 8 else (8, 5, 4)
    v, e, f, ld, lv = T.gen_cantilever(*dims, nen)
    ctx = T.Context(v, e, f, ld, lv, **KW, **TIGHT)
    orc = O.Oracle(v, e, f, ld, lv, **KW, **TIGHT)
    yield dict(T=T, O=O, ctx=ctx, orc=orc, v=v, e=e, f=f, nen=nen)
    ctx.close()
    orc.close()


def dev(cuda, a):
    return cuda.tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")


def host(t):
    return t.detach().cpu().numpy()


def test_element_matrices(pair):
    ctx, orc, e = pair["ctx"], pair["orc"], pair["e"]
    for el in [0, 1, 31, 32, e.shape[0] // 2, e.shape[0] - 1]:
        assert rel(ctx.element_matrix(el), orc.element_ke(el)) < 1e-12


def test_volumes(pair):
    vol, tv = pair["ctx"].volumes()
    otv, ovol = pair["orc"].total_volume()
    assert rel(host(vol), ovol) < 1e-14
    assert abs(tv - otv) <= 1e-12 * otv


def test_operator_apply(pair, cuda):
    """K(x) u with Dirichlet identity rows/columns (SolveFem.cpp:297-337)."""
    ctx, orc, e, v, f = pair["ctx"], pair["orc"], pair["e"], pair["v"], pair["f"]
    rng = np.random.default_rng(5)
    x = rng.uniform(0.01, 1.0, e.shape[0])
    u = rng.standard_normal(3 * v.shape[0])
    y = host(ctx.fem_apply(dev(cuda, x), dev(cuda, u)))
    orc.assemble(x)
    assert rel(y, orc.kmatvec(u)) < 1e-12
    assert np.array_equal(y[f], u[f])  # identity rows exactly


def test_solve_and_sensitivities(pair, cuda):
    ctx, orc, e = pair["ctx"], pair["orc"], pair["e"]
    x = np.random.default_rng(6).uniform(0.05, 1.0, e.shape[0])
    fx, gx, df, dg, rc = ctx.fem_obj_sens(dev(cuda, x))
    assert rc == 0
    U = host(ctx.displacement())
    ofx, ogx, odf, odg, oU = orc.fem_obj_sens(x, return_u=True)
    assert abs(fx - ofx) <= 1e-8 * abs(ofx)
    assert rel(U, oU) < 1e-7
    assert abs(gx[0] - ogx[0]) < 1e-12
    assert rel(host(df), odf) < 1e-7
    assert rel(host(dg), odg) < 1e-13
    info = ctx.info()
    assert info.fem_relres < 1e-9 and info.fem_status == 0


def test_filter_warm_start_sequence(pair, cuda):
    """Filter / ComputeFilteredSens share one warm-started CG state RX
    (PDEFilter.cpp:127): a sequence of calls must match the oracle's."""
    ctx, orc, e = pair["ctx"], pair["orc"], pair["e"]
    rng = np.random.default_rng(7)
    ctx.filter_state(dev(cuda, np.zeros(pair["v"].shape[0])))
    orc.filter_state(np.zeros(pair["v"].shape[0]))
    for _ in range(2):
        x = rng.uniform(0, 1, e.shape[0])
        assert rel(host(ctx.filter(dev(cuda, x), 0.01)), orc.filter(x, 0.01)) < 1e-9
        df = -rng.uniform(0, 5, e.shape[0])
        dg = rng.uniform(0, 1, e.shape[0])
        gdf, gdg = ctx.filter_sens(dev(cuda, df), dev(cuda, dg))
        odf, odg = orc.filter_sens(df, dg)
        assert rel(host(gdf), odf) < 1e-9
        assert rel(host(gdg), odg) < 1e-9
        assert rel(host(ctx.filter_state()), orc.filter_state()) < 1e-9


def test_heaviside_and_projected_sens(pair, cuda):
    ctx, orc, e = pair["ctx"], pair["orc"], pair["e"]
    rng = np.random.default_rng(8)
    xf = rng.uniform(0.01, 1, e.shape[0])
    for itr in (1, 29, 30, 40, 41, 50):
        xp = host(ctx.heaviside(dev(cuda, xf), itr, proj=1))
        oxp = orc.heaviside(xf, itr, proj=1)
        assert rel(xp, oxp) < 1e-14
        df, dg = rng.standard_normal(e.shape[0]), rng.standard_normal(e.shape[0])
        a, b = ctx.projected_sens(dev(cuda, xf), dev(cuda, df), dev(cuda, dg))
        oa, ob = orc.projected_sens(xf, df, dg)
        assert rel(host(a), oa) < 1e-14 and rel(host(b), ob) < 1e-14
    assert np.array_equal(host(ctx.heaviside(dev(cuda, xf), 3, proj=0)), xf)  # VecCopy


def test_mma_sequence(pair, cuda):
    """Successive MMA::Update calls (asymptote branches k < 3 and k > 2) and
    DesignChange against the oracle."""
    ctx, orc, e = pair["ctx"], pair["orc"], pair["e"]
    T, O = pair["T"], pair["O"]
    v = pair["v"]
    c2 = T.Context(v, e, pair["f"], np.array([3 * (v.shape[0] - 1) + 2], np.int32), np.array([-1.0]), **KW)
    o2 = O.Oracle(v, e, pair["f"], np.array([3 * (v.shape[0] - 1) + 2], np.int32), np.array([-1.0]), **KW)
    rng = np.random.default_rng(9)
    n = e.shape[0]
    x = rng.uniform(0.05, 0.6, n)
    xold = x.copy()
    for it in range(4):
        df = -rng.uniform(0.1, 3.0, n)
        dg = rng.uniform(0.5, 1.5, n) / n
        gx = np.array([x.mean() - 0.3])
        gmn, gmx = c2.mma_movelimit(dev(cuda, x))
        omn, omx = o2.mma_movelimit(x)
        assert np.array_equal(host(gmn), omn) and np.array_equal(host(gmx), omx)
        xn = host(c2.mma_update(dev(cuda, x), dev(cuda, df), gx, dev(cuda, dg), gmn, gmx))
        oxn = o2.mma_update(x, df, gx, dg, omn, omx)
        assert rel(xn, oxn) < 1e-8, it
        assert np.all(xn >= omn - 1e-15) and np.all(xn <= omx + 1e-15)
        ch, _ = c2.mma_design_change(dev(cuda, oxn), dev(cuda, xold))
        och, _ = o2.mma_design_change(oxn, xold)
        assert abs(ch - och) < 1e-15
        xold, x = x, oxn
    xo1, xo2, L, U, k = c2.mma_state()
    oxo1, oxo2, oL, oU, ok = o2.mma_state()
    assert k == ok == 4
    assert rel(host(xo1), oxo1) < 1e-12 and rel(host(L), oL) < 1e-8 and rel(host(U), oU) < 1e-8
    c2.close()
    o2.close()
