"""bench.py's roofline byte model on CPU: the inputs it derives from the
mesh and the per-launch byte formulas of the kernels it reports."""
import sys

from conftest import ROOT


def test_roofline_byte_model_inputs(T, O):
    """The roofline's byte model: the level-0 block count bench.py derives
    from the connectivity equals the oracle's assembled operator (9 scalar
    entries per 3x3 block), and the per-launch byte formulas follow the
    stated per-element / per-node terms."""
    import types
    import numpy as np
    sys.path.insert(0, ROOT)
    import bench
    v, e, f, ld, lv = T.gen_cantilever(8, 5, 4, 8)
    orc = O.Oracle(v, e, f, ld, lv, Emax=1.0, rmin=1.5)
    orc.assemble(np.full(e.shape[0], 0.5))
    K = orc.csr()
    nnzb = bench._graph_nnzb(e, v.shape[0])
    pairs = {(int(a), int(b)) for el in e for a in el for b in el}
    assert nnzb == len(pairs)
    # every stored entry of the assembled operator lies in one of those blocks;
    # Dirichlet rows and columns may store fewer (identity rows)
    rows, cols = K.nonzero()
    assert {(int(i) // 3, int(j) // 3) for i, j in zip(rows, cols)} <= pairs
    assert K.nnz <= 9 * nnzb
    ctx = types.SimpleNamespace(nen=8, ne=e.shape[0], nn=v.shape[0], ndof=3 * v.shape[0])
    assert bench.kmv_bytes(ctx, 8) == ctx.ne * (32 + 4 + 8 + 2400) + ctx.nn * 3 * 16
    assert bench.cheb0_bytes(ctx, nnzb, 4) == nnzb * 40 + (ctx.nn + 1) * 4 + ctx.ndof * 28
    orc.close()
