"""GPU parity on the benchmark configurations' own shapes, through the C ABI,
against the CPU oracle on the same seeded inputs.

- the tightly converged FP64 solve (U within 1e-7, compliance within 1e-8,
  dfdx within 1e-7 relative, gx within 1e-12) on the 40 x 20 x 10 hex8
  cantilever (8,000 elements, the plain-method configuration) and on a
  20 x 10 x 6 tet4 box (7,200 tets, interior nodes jittered by +-0.2 h);
- the design loop with Heaviside projection on (proj = 1), 45 iterations, so
  that beta steps at iterations 30 and 40 (PDEFilter.cpp:242-293) and the
  projected sensitivities feed the filter and MMA (main.cpp:88-107); bar: the
  trajectory bar of the plain loop (final compliance within 1e-3 relative);
- MMA's secondary paths: SetAsymptotes, RobustAsymptotesType = 1
  (MMA.cpp:561-575), constraintModification (MMA.cpp:590-596), the
  KKTresidual (MMA.cpp:412-480) after each update, and a restart from the
  exported history (MMA.cpp:91-176, 302-342);
- the reference's own boundary-condition files (mesh/fixeddofs.txt,
  loaddof_1.txt, load_1.txt: 8733 clamped DOFs, 41 unit loads) read through
  topo_read_mesh_dir and solved on the 140 x 70 x 40 lattice (392,000 hex8),
  checked by the energy identity sum_e E_e u_e'Ke u_e = F'U;
- a mesh written in the reference's text formats and read back runs the same
  trajectory as the generator's arrays;
- the main.cpp-shaped C++ program (include/topopt.hpp) run on the GPU
  against the oracle's loop.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, rel

pytestmark = pytest.mark.gpu

KW = dict(Emax=1.0, rmin=1.5, volfrac=0.12)
TIGHT = dict(fem_rtol=1e-10, filter_rtol=1e-12)


def dev(cuda, a):
    return cuda.tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")


@pytest.mark.parametrize("nen,dims", [(8, (40, 20, 10)), (4, (20, 10, 6))], ids=["hex8-40x20x10", "tet4-20x10x6"])
def test_tight_solve_and_sensitivities(T, O, cuda, nen, dims):
    v, e, f, ld, lv = T.gen_cantilever(*dims, nen)
    v2, e2, f2, ld2, lv2 = O.cantilever(*dims, elem="hex8" if nen == 8 else "tet4")
    assert np.array_equal(v, v2) and np.array_equal(e, e2) and np.array_equal(f, f2)
    ctx = T.Context(v, e, f, ld, lv, **KW, **TIGHT)
    orc = O.Oracle(v, e, f, ld, lv, **KW, **TIGHT)
    x = np.random.default_rng(21).uniform(0.05, 1.0, e.shape[0])
    fx, gx, df, dg, rc = ctx.fem_obj_sens(dev(cuda, x))
    assert rc == 0 and ctx.info().fem_relres < 1e-9
    ofx, ogx, odf, odg, oU = orc.fem_obj_sens(x, return_u=True)
    assert abs(fx - ofx) <= 1e-8 * abs(ofx)
    assert rel(ctx.displacement().cpu().numpy(), oU) < 1e-7
    assert rel(df.cpu().numpy(), odf) < 1e-7
    assert abs(gx[0] - ogx[0]) < 1e-12
    assert rel(dg.cpu().numpy(), odg) < 1e-13
    ctx.close()
    orc.close()


def test_projection_loop_45_iterations(T, O, cuda):
    v, e, f, ld, lv = T.gen_cantilever(40, 20, 10, 8)
    kw = dict(KW, proj=1, fem_rtol=1e-5)
    ctx = T.Context(v, e, f, ld, lv, ch_tol=0.0, **kw)
    ctx.opt_init()
    hist = ctx.opt_run(45)
    orc = O.Oracle(v, e, f, ld, lv, **kw)
    ohist, oxp = orc.run(45, ch_tol=0.0)
    assert hist.shape == (45, 3) and ohist.shape == (45, 3)
    relf = np.abs(hist[:, 0] - ohist[:, 0]) / np.abs(ohist[:, 0])
    assert relf[-1] < 1e-3, relf
    assert relf.max() < 5e-3, relf
    assert np.abs(hist[:, 1] - ohist[:, 1]).max() < 1e-3
    xp = ctx.opt_tensor(1).cpu().numpy()
    assert xp.min() >= 0.01 - 1e-15 and xp.max() <= 1.0
    assert np.abs(xp - oxp).max() < 5e-2
    ctx.close()
    orc.close()


def test_mma_options_kkt_and_restart(T, O, cuda):
    v, e, f, ld, lv = T.gen_cantilever(12, 6, 4, 8)
    opts = dict(asyminit=0.4, asymdec=0.65, asyminc=1.15, robust=1, constraint_mod=1)
    ctx = T.Context(v, e, f, ld, lv, **KW)
    orc = O.Oracle(v, e, f, ld, lv, **KW)
    ctx.mma_options(**opts)
    orc.mma_options(**opts)
    n = e.shape[0]
    rng = np.random.default_rng(31)
    x = rng.uniform(0.05, 0.6, n)
    inputs, outs, snap = [], [], None
    for it in range(6):
        df = -rng.uniform(0.1, 3.0, n)
        dg = rng.uniform(0.5, 1.5, n) / n
        gx = np.array([x.mean() - 0.3])
        gmn, gmx = ctx.mma_movelimit(dev(cuda, x))
        omn, omx = orc.mma_movelimit(x)
        xn = ctx.mma_update(dev(cuda, x), dev(cuda, df), gx, dev(cuda, dg), gmn, gmx).cpu().numpy()
        oxn = orc.mma_update(x, df, gx, dg, omn, omx)
        assert rel(xn, oxn) < 1e-8, it
        n2, ni = ctx.mma_kkt(dev(cuda, oxn), dev(cuda, df), gx, dev(cuda, dg), gmn, gmx)
        on2, oni = orc.mma_kkt(oxn, df, gx, dg, omn, omx)
        assert abs(n2 - on2) <= 1e-6 * on2 and abs(ni - oni) <= 1e-6 * oni, (it, n2, on2, ni, oni)
        inputs.append((x, df, dg, gx))
        outs.append(oxn)
        if it == 2:
            snap = ctx.mma_state()
            assert snap[4] == 3
        x = oxn
    # restart at k = 3 from the exported history, on a fresh context and a
    # fresh oracle, with the same options: updates 4..6 repeat exactly
    xo1, xo2, L, U, k = snap
    c2 = T.Context(v, e, f, ld, lv, **KW)
    o2 = O.Oracle(v, e, f, ld, lv, **KW)
    c2.mma_options(**opts)
    o2.mma_options(**opts)
    c2.mma_restart_set(xo1, xo2, U, L, k)
    o2.mma_restart_set(xo1.cpu().numpy(), xo2.cpu().numpy(), U.cpu().numpy(), L.cpu().numpy(), k)
    for it in range(3, 6):
        x, df, dg, gx = inputs[it]
        gmn, gmx = c2.mma_movelimit(dev(cuda, x))
        xn = c2.mma_update(dev(cuda, x), dev(cuda, df), gx, dev(cuda, dg), gmn, gmx).cpu().numpy()
        omn, omx = o2.mma_movelimit(x)
        oxn = o2.mma_update(x, df, gx, dg, omn, omx)
        assert rel(xn, outs[it]) < 1e-8 and rel(oxn, outs[it]) < 1e-12, it
    for h in (ctx, c2, orc, o2):
        h.close()


def test_reference_bc_files_solved_at_392k(T, cuda, tmp_path):
    """The reference's 8733 fixed DOFs and 41 unit loads (its own files,
    read through topo_read_mesh_dir) on the 140 x 70 x 40 lattice: the solve
    converges and the compliance equals F'U (energy identity of K U = F with
    the Dirichlet rows as identity), within the solve tolerance."""
    from test_host import read_reference_bcs
    _, _, f, ld, lv, _ = read_reference_bcs(T, tmp_path)
    v, e, _, _, _ = T.gen_cantilever(140, 70, 40, 8)
    assert 3 * v.shape[0] > max(f.max(), ld.max())
    ctx = T.Context(v, e, f, ld, lv, precision=T.PREC_MIXED, fem_rtol=1e-8, **KW)
    x = dev(cuda, np.random.default_rng(41).uniform(0.1, 1.0, e.shape[0]))
    fx, gx, df, dg, rc = ctx.fem_obj_sens(x)
    assert rc == 0 and ctx.info().fem_relres < 1e-8
    U = ctx.displacement().cpu().numpy()
    assert np.abs(U[f]).max() <= 1e-12 * np.abs(U).max()
    fu = float(np.dot(lv, U[ld]))
    assert fx > 0 and abs(fx - fu) <= 1e-6 * fu
    d = df.cpu().numpy()
    assert np.all(np.isfinite(d)) and d.max() <= 0.0
    ctx.close()


def test_mesh_files_run_like_the_generator_arrays(T, cuda, tmp_path):
    v, e, f, ld, lv = T.gen_cantilever(16, 8, 6, 8)
    np.savetxt(tmp_path / "vertex.txt", v, fmt="%.17g")
    np.savetxt(tmp_path / "element.txt", e, fmt="%d")
    np.savetxt(tmp_path / "fixeddofs.txt", f, fmt="%d")
    np.savetxt(tmp_path / "loaddof_1.txt", ld[None, :], fmt="%d", delimiter="\t")
    np.savetxt(tmp_path / "load_1.txt", lv[None, :], fmt="%.17g", delimiter="\t")
    rv, re_, rf, rld, rlv, cp = T.read_mesh_dir(str(tmp_path), 8, 1)
    h = []
    for arrays in ((v, e, f, ld, lv), (rv, re_, rf, rld, rlv)):
        ctx = T.Context(*arrays, ch_tol=0.0, **KW)
        ctx.opt_init()
        h.append(ctx.opt_run(4))
        ctx.close()
    # the element scatter's float atomics leave rounding-level differences between two contexts
    assert rel(h[1][:, 0], h[0][:, 0]) < 1e-6 and np.abs(h[1][:, 1] - h[0][:, 1]).max() < 1e-9


def test_cpp_driver_program_matches_the_oracle_loop(T, O, cuda, tmp_path):
    """host/topopt_main.cpp (the main.cpp loop over the reference-shaped C++
    classes of include/topopt.hpp) on the GPU: its printed `It.: ... fx:`
    trajectory against the oracle's loop (main.cpp:70-119), same bar as the
    library's own loop."""
    exe = os.path.join(ROOT, "unstructured-fea-based-topology-optimization-in-petsc-and-eigen_b200", "topopt")
    r = subprocess.run([exe, "-lattice", "40", "20", "10", "-Emax", "1", "-rmin", "1.5", "-maxItr", "20",
                        "-ch_tol", "0", "-vtu", str(tmp_path)], cwd=tmp_path, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    fx = [float(line.split("fx:")[1].split(",")[0]) for line in r.stdout.splitlines() if line.startswith("It.:")]
    assert len(fx) == 20
    assert (tmp_path / "output_final.vtu").exists() and (tmp_path / "output_20.vtu").exists()
    v, e, f, ld, lv = T.gen_cantilever(40, 20, 10, 8)
    orc = O.Oracle(v, e, f, ld, lv, **KW)
    ohist, _ = orc.run(20, ch_tol=0.0)
    relf = np.abs(np.array(fx) - ohist[:, 0]) / np.abs(ohist[:, 0])
    assert relf[-1] < 1e-3 and relf.max() < 5e-3, relf
    orc.close()
