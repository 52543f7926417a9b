"""The allocation-free sensitivity entry point (topo_fem_sensitivities_noalloc)
for callers that cannot allocate device memory when they need the
reduction, checked through the C ABI against the existing entry point
(topo_fem_obj_sens) and against the oracle's sums for the same
displacement (SolveFem.cpp:208-249), on two calls in a row: the second call
must not see the first call's leftovers in the shared scratch.  A mesh of
about 1e5 elements spreads the reduction over hundreds of blocks.  This file
is collected last on purpose; it passes alone in a fresh process as well."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KW = dict(Emax=1.0, rmin=1.5, volfrac=0.12, fem_rtol=1e-8)


def packed(ke):
    n = ke.shape[0]
    return np.concatenate([ke[i, i:] for i in range(n)])


@pytest.mark.parametrize("nen", [8, 4])
def test_noalloc_matches_obj_sens_twice(T, O, cuda, nen):
    dims = (14, 7, 5) if nen == 8 else (7, 4, 3)
    v, e, f, ld, lv = T.gen_cantilever(*dims, nen)
    ctx = T.Context(v, e, f, ld, lv, **KW)
    orc = O.Oracle(v, e, f, ld, lv, **KW)
    ne = e.shape[0]
    ke = np.stack([packed(ctx.element_matrix(i)) for i in range(ne)])
    vol, tv = ctx.volumes()
    dev = lambda a, dt=cuda.float64: cuda.tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")
    e_d, ke_d = dev(e.ravel(), cuda.int32), dev(ke.ravel())
    ptr = lambda t: C.c_void_p(t.data_ptr())
    rng = np.random.default_rng(31)
    for call in range(2):
        x = rng.uniform(0.05, 1.0, ne)
        x_d = dev(x)
        fx, gx, df, dg, rc = ctx.fem_obj_sens(x_d)
        assert rc == 0
        U = ctx.displacement()
        df2, dg2, out = cuda.zeros(ne, dtype=cuda.float64, device="cuda"), \
            cuda.zeros(ne, dtype=cuda.float64, device="cuda"), cuda.zeros(2, dtype=cuda.float64, device="cuda")
        cuda.cuda.synchronize()
        rc = T.lib().topo_fem_sensitivities_noalloc(nen, ne, ptr(e_d), ptr(ke_d), ptr(x_d), ptr(vol), ptr(U), 1e-9,
                                                     1.0, 3.0, tv, 0.12, ptr(df2), ptr(dg2), ptr(out), None)
        assert rc == 0, T.last_error()
        cuda.cuda.synchronize()
        o = out.cpu().numpy()
        assert abs(o[0] - fx) <= 1e-12 * abs(fx), call
        assert abs(o[1] - gx[0]) <= 1e-12, call
        assert np.abs(df2.cpu().numpy() - df.cpu().numpy()).max() <= 1e-12 * np.abs(df.cpu().numpy()).max(), call
        assert np.abs(dg2.cpu().numpy() - dg.cpu().numpy()[0]).max() <= 1e-15, call
        # the oracle builds its own element matrices, which agree with the
        # library's to 1e-12 per entry (the element parity bar); u'Ke u
        # amplifies that by its cancellation, hence 1e-10 here
        ofx, ogx, odf, odg = orc.obj_sens_given_u(x, U.cpu().numpy())
        assert abs(o[0] - ofx) <= 1e-10 * abs(ofx) and abs(o[1] - ogx[0]) <= 1e-12, call
        assert np.abs(df2.cpu().numpy() - odf).max() <= 1e-10 * np.abs(odf).max(), call
        assert np.abs(dg2.cpu().numpy() - odg[0]).max() <= 1e-15, call
    ctx.close()
    orc.close()


def test_noalloc_many_blocks_against_the_oracle(T, O, cuda):
    """98,304 hex8 elements (768 blocks of the per-call reduction): two calls
    in a row with different displacements, against the oracle."""
    v, e, f, ld, lv = O.cantilever(64, 32, 48, elem="hex8")
    ne = e.shape[0]
    orc = O.Oracle(v, e, f, ld, lv, **KW)
    ke = np.stack([packed(orc.element_ke(i)) for i in range(ne)])
    tv, vol = orc.total_volume()
    dev = lambda a, dt=cuda.float64: cuda.tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")
    ptr = lambda t: C.c_void_p(t.data_ptr())
    e_d, ke_d, vol_d = dev(e.ravel(), cuda.int32), dev(ke.ravel()), dev(vol)
    rng = np.random.default_rng(32)
    for call in range(2):
        x = rng.uniform(0.01, 1.0, ne)
        U = rng.standard_normal(3 * v.shape[0]) * (1.0 + call)
        x_d, U_d = dev(x), dev(U)
        df, dg, out = [cuda.zeros(k, dtype=cuda.float64, device="cuda") for k in (ne, ne, 2)]
        cuda.cuda.synchronize()
        rc = T.lib().topo_fem_sensitivities_noalloc(8, ne, ptr(e_d), ptr(ke_d), ptr(x_d), ptr(vol_d), ptr(U_d), 1e-9,
                                                     1.0, 3.0, tv, 0.12, ptr(df), ptr(dg), ptr(out), None)
        assert rc == 0, T.last_error()
        cuda.cuda.synchronize()
        ofx, ogx, odf, odg = orc.obj_sens_given_u(x, U)
        o = out.cpu().numpy()
        assert abs(o[0] - ofx) <= 1e-12 * abs(ofx), call
        assert abs(o[1] - ogx[0]) <= 1e-12, call
        assert np.abs(df.cpu().numpy() - odf).max() <= 1e-12 * np.abs(odf).max(), call
        assert np.abs(dg.cpu().numpy() - odg[0]).max() <= 1e-15, call
    orc.close()


def test_noalloc_rejects_oversize(T, cuda):
    rc = T.lib().topo_fem_sensitivities_noalloc(8, 2_000_000, C.c_void_p(1), C.c_void_p(1), C.c_void_p(1),
                                                 C.c_void_p(1), C.c_void_p(1), 1e-9, 1.0, 3.0, 1.0, 0.1,
                                                 C.c_void_p(1), C.c_void_p(1), C.c_void_p(1), None)
    assert rc == -1 and "at most" in T.last_error()
