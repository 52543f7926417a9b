"""k-load block path (load cases sharing one stiffness matrix; compliance and
its sensitivity summed over the cases) through the C ABI.

The oracle solves one load case per context (the reference assembles its
NUM_LD loads into one F, SolveFem.cpp:277-282, so a case is one oracle
context); the block results are checked against the per-case oracle
solutions summed over the cases, and against the library's own one-by-one
path (`fem_block = 0`).

Tolerances (FP64): block operator 1e-12 relative per case (summation order
only); tightly converged solves (rtol 1e-10): compliance 1e-8, displacements
1e-7, sensitivities 1e-7 relative; block against one-by-one at rtol 1e-5:
compliance 1e-6 relative."""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

KW = dict(Emax=1.0, rmin=1.5, volfrac=0.12)
TIGHT = dict(fem_rtol=1e-10, filter_rtol=1e-12)


def dev(cuda, a):
    return cuda.tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")


def host(t):
    return t.detach().cpu().numpy()


def mesh(T, nen, k):
    dims = (12, 6, 6) if nen == 8 else (6, 4, 4)
    v, e, f, _, _ = T.gen_cantilever(*dims, nen)
    ld, lv = T.gen_multiload(*dims, k)
    cp = np.arange(0, 3 * k + 1, 3, dtype=np.int32)
    return v, e, f, ld, lv, cp


@pytest.mark.parametrize("stages", [2, 3])
@pytest.mark.parametrize("nen,k", [(8, 3), (8, 8), (8, 11), (4, 3), (4, 8)])
def test_block_operator_matches_oracle(T, O, cuda, nen, k, stages):
    """K(x) [u_1..u_k] by the tensor-core block kernel (2 and 3 element-matrix
    copies in flight per warp) against the oracle's assembled K applied case
    by case (Dirichlet rows/columns identity)."""
    v, e, f, ld, lv, cp = mesh(T, nen, k)
    ctx = T.Context(v, e, f, ld, lv, case_ptr=cp, blk_stages=stages, **KW)
    orc = O.Oracle(v, e, f, ld[:3], lv[:3], **KW)
    rng = np.random.default_rng(11 + k)
    x = rng.uniform(0.01, 1.0, e.shape[0])
    U = rng.standard_normal((k, 3 * v.shape[0]))
    Y = host(ctx.fem_apply_block(dev(cuda, x), dev(cuda, U.ravel()))).reshape(k, -1)
    orc.assemble(x)
    for c in range(k):
        assert rel(Y[c], orc.kmatvec(U[c])) < 1e-12, c
        assert np.array_equal(Y[c][f], U[c][f])  # identity rows exactly
    ctx.close()
    orc.close()


@pytest.mark.parametrize("nen,k", [(8, 3), (8, 8), (4, 3)])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_block_solve_matches_per_case_oracle(T, O, cuda, nen, k, prec):
    v, e, f, ld, lv, cp = mesh(T, nen, k)
    ctx = T.Context(v, e, f, ld, lv, case_ptr=cp, precision=T.PREC_MIXED if prec == "mixed" else T.PREC_FP64,
                    **KW, **TIGHT)
    rng = np.random.default_rng(3)
    x = rng.uniform(0.05, 1.0, e.shape[0])
    fx, gx, df, dg, rc = ctx.fem_obj_sens(dev(cuda, x))
    assert rc == 0
    info = ctx.info()
    assert info.fem_status == 0 and info.fem_relres < 1e-9
    U = host(ctx.displacement()).reshape(k, -1)
    ofx, odf = 0.0, np.zeros(e.shape[0])
    for c in range(k):
        orc = O.Oracle(v, e, f, ld[cp[c]:cp[c + 1]], lv[cp[c]:cp[c + 1]], **KW, **TIGHT)
        fxc, gxc, dfc, dgc, Uc = orc.fem_obj_sens(x, return_u=True)
        ofx += fxc
        odf += dfc
        assert rel(U[c], Uc) < 1e-7, c
        if c == 0:
            assert abs(gx[0] - gxc[0]) < 1e-12 and rel(host(dg), dgc) < 1e-13
        orc.close()
    assert abs(fx - ofx) <= 1e-8 * abs(ofx)
    assert rel(host(df), odf) < 1e-7
    ctx.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_block_equals_one_by_one(T, cuda, prec):
    """The lockstep block solve and the case-by-case solve meet the same
    stopping rule (rtol 1e-5 per case) and agree on compliance."""
    v, e, f, ld, lv, cp = mesh(T, 8, 8)
    out = []
    for blk in (1, 0):
        ctx = T.Context(v, e, f, ld, lv, case_ptr=cp, fem_block=blk,
                        precision=T.PREC_MIXED if prec == "mixed" else T.PREC_FP64, **KW)
        x = np.full(e.shape[0], 0.12)
        fx, gx, df, dg, rc = ctx.fem_obj_sens(dev(cuda, x))
        assert rc == 0 and ctx.info().fem_relres < 1e-5
        out.append((fx, host(df)))
        ctx.close()
    assert abs(out[0][0] - out[1][0]) <= 1e-6 * abs(out[1][0])
    assert rel(out[0][1], out[1][1]) < 1e-4


def test_block_design_loop(T, cuda):
    """Ten design iterations, block against one-by-one (mixed precision)."""
    v, e, f, ld, lv, cp = mesh(T, 8, 4)
    hist = []
    for blk in (1, 0):
        ctx = T.Context(v, e, f, ld, lv, case_ptr=cp, fem_block=blk, precision=T.PREC_MIXED, ch_tol=0.0, **KW)
        ctx.opt_init()
        h = ctx.opt_run(10)
        hist.append(h)
        ctx.close()
    assert rel(hist[0][:, 0], hist[1][:, 0]) < 1e-4
    assert np.abs(hist[0][:, 1] - hist[1][:, 1]).max() < 1e-4


def test_block_graph_replay_matches_direct(T, cuda):
    """The block FGMRES steps replayed from CUDA graphs reproduce the directly
    launched design trajectory."""
    v, e, f, ld, lv, cp = mesh(T, 8, 8)
    hist = []
    for g in (1, 0):
        ctx = T.Context(v, e, f, ld, lv, case_ptr=cp, fem_graphs=g, precision=T.PREC_MIXED, ch_tol=0.0, **KW)
        ctx.opt_init()
        hist.append(ctx.opt_run(6))
        ctx.close()
    assert rel(hist[0][:, 0], hist[1][:, 0]) < 1e-6
