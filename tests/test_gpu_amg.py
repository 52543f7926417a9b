"""The device-built smoothed-aggregation hierarchy (the numeric Galerkin
products recomputed every design iteration) against scipy algebra on the
matrices the device returns, and the level-0 operator against the oracle's
assembled K."""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[0, 1], ids=["fp64", "mixed"])
def built(request, T, O, cuda):
    v, e, f, ld, lv = T.gen_cantilever(24, 12, 8, 8)
    prec = request.param
    ctx = T.Context(v, e, f, ld, lv, Emax=1.0, rmin=1.5, precision=prec, fem_rtol=1e-8)
    x = np.random.default_rng(21).uniform(0.01, 1.0, e.shape[0])
    U, rc = ctx.fem_solve(cuda.tensor(x, device="cuda"))
    assert rc == 0
    orc = O.Oracle(v, e, f, ld, lv, Emax=1.0, rmin=1.5)
    orc.assemble(x)
    yield ctx, orc, prec
    ctx.close()


def test_level0_is_assembled_K(built):
    ctx, orc, prec = built
    A0 = ctx.amg_level(0, 0)
    K = orc.csr()
    tol = 1e-13 if prec == 0 else 2e-7
    assert abs(A0 - K).max() <= tol * abs(K).max()


def test_galerkin_products(built):
    ctx, _, prec = built
    info = ctx.info()
    tol = 1e-12 if prec == 0 else 1e-5
    for l in range(info.amg_levels - 1):
        A = ctx.amg_level(l, 0)
        P = ctx.amg_level(l, 1)
        R = ctx.amg_level(l, 2)
        Ac = ctx.amg_level(l + 1, 0)
        assert abs(R - P.T).max() == 0.0  # numeric transpose is exact
        ref = (P.T @ A @ P).tocsr()
        assert abs(Ac - ref).max() <= tol * abs(ref).max(), l
        assert Ac.shape[0] == info.amg_dofs[l + 1]


def test_prolongator_structure(built):
    """Level-0 P (smoothed aggregation) has one 3 x 6 block per (node,
    neighbouring aggregate) and reproduces the rigid-body translations away
    from the clamped face: P applied to the coarse translation modes equals
    the fine translation up to the smoothing correction, which vanishes where
    D^-1 A annihilates translations (interior rows of unconstrained nodes)."""
    ctx, _, prec = built
    P = ctx.amg_level(0, 1)
    A = ctx.amg_level(0, 0)
    assert np.isfinite(P.data).all() and P.shape[1] % 6 == 0
    nagg = P.shape[1] // 6
    assert nagg == ctx.info().amg_dofs[1] // 6
    # A annihilates rigid translations in rows whose stencil touches no fixed DOF
    t = np.tile([1.0, 0.0, 0.0], A.shape[0] // 3)
    At = A @ t
    rows_free = np.abs(At) < (1e-9 if prec == 0 else 1e-5) * abs(A).max()
    assert rows_free.mean() > 0.5


def test_cluster_coarse_cycle_matches_per_level_kernels(T, cuda):
    """The lower V-cycle run by one thread-block cluster gives the same solve
    (same operations, summation order aside) as the per-level kernels."""
    import numpy as np
    v, e, f, ld, lv = T.gen_cantilever(40, 20, 10, 8)
    x = cuda.tensor(np.random.default_rng(4).uniform(0.05, 1.0, e.shape[0]), device="cuda")
    out = []
    for cc in (1, 0):
        ctx = T.Context(v, e, f, ld, lv, Emax=1.0, rmin=1.5, volfrac=0.12, amg_coarse_cta=cc, fem_rtol=1e-8)
        fx, gx, df, dg, rc = ctx.fem_obj_sens(x)
        assert rc == 0
        out.append((fx, ctx.info().fem_its))
        ctx.close()
    assert abs(out[0][0] - out[1][0]) <= 1e-10 * abs(out[1][0])
    assert abs(out[0][1] - out[1][1]) <= 1
