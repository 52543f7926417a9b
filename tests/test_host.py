"""Host-side logic and the C-ABI boundary, without a GPU: the library loads,
exports every symbol include/topo.h declares, its host routines (mesh
generator, graph aggregation, mesh-file reader, argument validation) agree
with the oracle and fail loudly on bad input."""
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "topo.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(topo_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol(T):
    L = T.lib()
    syms = header_symbols()
    assert len(syms) >= 40
    for s in syms:
        assert hasattr(L, s), s
    assert sorted(T.symbols()) == syms  # the ctypes bindings cover the header exactly


def test_version_and_defaults(T):
    assert b"sm_100a" in T.lib().topo_version()
    p = T.default_params()
    # OptPara.cpp:66-78, SolveFem.cpp:11,134, PDEFilter.cpp:117-120
    assert (p.Emin, p.Emax, p.volfrac, p.penal, p.rmin, p.Xmin, p.Xmax, p.movlim) == \
        (1e-9, 1e6, 0.12, 3.0, 0.01, 0.01, 1.0, 0.2)
    assert (p.x0, p.beta0, p.betamax, p.proj, p.maxItr, p.m, p.nu) == (0.5, 1.0, 8.0, 0, 200, 1, 0.3)
    assert (p.fem_rtol, p.filter_rtol, p.filter_atol, p.filter_dtol, p.filter_maxit) == (1e-5, 1e-5, 1e-50, 1e5, 10000)


def test_struct_mirrors_match_the_library(T):
    """The ctypes mirrors of topo_params / topo_solve_info have the library's
    sizes, and topo_params_default writes exactly sizeof(topo_params) bytes
    (a guard region after the struct stays untouched) with the solver
    defaults in the last fields."""
    import ctypes as C
    pb, ib = C.c_size_t(), C.c_size_t()
    assert T.lib().topo_struct_sizes(C.byref(pb), C.byref(ib)) == 0
    assert pb.value == C.sizeof(T.Params) and ib.value == C.sizeof(T.SolveInfo)
    buf = (C.c_ubyte * (pb.value + 64))(*([0xAB] * (pb.value + 64)))
    T.lib().topo_params_default(C.cast(buf, C.POINTER(T.Params)))
    assert bytes(buf[pb.value:]) == b"\xab" * 64
    p = T.Params.from_buffer(buf)
    assert (p.cheb_degree, p.cheb_degree_post, p.cheb_degree_coarse) == (2, 0, 4)
    assert (p.fem_restart, p.fem_block, p.fem_graphs, p.autotune, p.pdl) == (30, 1, 1, 1, 1)
    assert (p.amg_coarse_cta, p.amg_half_fine, p.fem_warm_start) == (0, 0, 0)
    assert (p.step_graph, p.blk_stages, p.deterministic) == (0, 0, 0)


@pytest.mark.parametrize("nen", [8, 4])
def test_generator_matches_oracle_bit_exact(T, O, nen):
    v, e, f, ld, lv = T.gen_cantilever(9, 5, 4, nen)
    v2, e2, f2, ld2, lv2 = O.cantilever(9, 5, 4, elem="hex8" if nen == 8 else "tet4")
    for a, b in [(v, v2), (e, e2), (f, f2), (ld, ld2), (lv, lv2)]:
        assert np.array_equal(a, b)
    m1 = T.gen_multiload(9, 5, 4, 8)
    m2 = O.multiload(9, 5, 4, 8)
    assert np.array_equal(m1[0], m2[0]) and np.array_equal(m1[1], m2[1])


def test_generator_lattice_layout(T):
    nx, ny, nz = 5, 3, 2
    v, e, f, ld, lv = T.gen_cantilever(nx, ny, nz, 8, jitter=0.0)
    assert v.shape == ((nx + 1) * (ny + 1) * (nz + 1), 3) and e.shape == (nx * ny * nz, 8)
    # diagonal local numbering: local l = a + 2b + 4c -> offset (a, b, c)
    co = v[e[0]]
    assert np.array_equal(co, [[l & 1, (l >> 1) & 1, (l >> 2) & 1] for l in range(8)])
    # x = 0 face clamped, unit total -z load on the x = L, z = 0 edge
    assert f.size == 3 * (ny + 1) * (nz + 1) and np.all(v[f // 3, 0] == 0)
    assert np.all(ld % 3 == 2) and abs(lv.sum() + 1.0) < 1e-15
    assert np.all(v[ld // 3, 0] == nx) and np.all(v[ld // 3, 2] == 0)


def test_aggregation_matches_oracle(T, O):
    """Integer work, compared bit-exactly: the library's greedy aggregation of
    the level-0 node graph equals the oracle's."""
    v, e, f, ld, lv = T.gen_cantilever(14, 7, 5, 8)
    orc = O.Oracle(v, e, f, ld, lv, Emax=1.0, rmin=1.5)
    orc.assemble(np.full(e.shape[0], 0.5))
    na_o, agg_o = orc.amg_aggregates(0)
    nn = v.shape[0]
    # node graph from the mesh (self included, sorted)
    nbr = [set() for _ in range(nn)]
    for el in e:
        for a in el:
            nbr[a].update(el.tolist())
    rp = np.zeros(nn + 1, dtype=np.int32)
    rp[1:] = np.cumsum([len(s) for s in nbr])
    ci = np.concatenate([sorted(s) for s in nbr]).astype(np.int32)
    fixed_nodes = np.zeros(nn, dtype=np.uint8)
    fixed_nodes[np.unique(f // 3)] = 1
    na, agg = T.graph_aggregate(rp, ci, fixed_nodes)
    agg_o = agg_o[:nn].copy()
    agg_o[agg_o == -2] = -1
    assert na == na_o
    assert np.array_equal(agg, agg_o)
    assert np.all(agg[fixed_nodes == 1] == -1)
    sizes = np.bincount(agg[agg >= 0])
    assert sizes.min() >= 2 and abs(sizes.mean() - 27) < 12


def test_mesh_dir_roundtrip(T, tmp_path):
    v, e, f, ld, lv = T.gen_cantilever(3, 2, 2, 8)
    np.savetxt(tmp_path / "vertex.txt", v, fmt="%.17g")
    np.savetxt(tmp_path / "element.txt", e, fmt="%d")
    np.savetxt(tmp_path / "fixeddofs.txt", f, fmt="%d")
    np.savetxt(tmp_path / "loaddof_1.txt", ld[None, :], fmt="%d", delimiter="\t")
    np.savetxt(tmp_path / "load_1.txt", lv[None, :], fmt="%.17g", delimiter="\t")
    v2, e2, f2, ld2, lv2, cp = T.read_mesh_dir(str(tmp_path), 8, 1)
    assert np.array_equal(v, v2) and np.array_equal(e, e2) and np.array_equal(f, f2)
    assert np.array_equal(ld, ld2) and np.array_equal(lv, lv2) and list(cp) == [0, ld.size]
    with pytest.raises(T.TopoError) as ei:
        T.read_mesh_dir(str(tmp_path / "missing"), 8, 1)
    assert ei.value.code == -8  # TOPO_ERR_IO ("Can't found document")


REF_MESH = os.path.join(ROOT, "tests", "golden", "reference_mesh")


def read_reference_bcs(T, tmp_path):
    """The reference's own boundary-condition files (mesh/fixeddofs.txt,
    loaddof_1.txt, load_1.txt, copied byte for byte by
    tests/golden/make_golden.py) read through topo_read_mesh_dir, beside a
    one-element vertex/element pair (the reference's mesh blobs are not
    in its repository)."""
    import shutil
    for name in ("fixeddofs.txt", "loaddof_1.txt", "load_1.txt"):
        shutil.copyfile(os.path.join(REF_MESH, name), tmp_path / name)
    v, e, _, _, _ = T.gen_cantilever(1, 1, 1, 8)
    np.savetxt(tmp_path / "vertex.txt", v, fmt="%.17g")
    np.savetxt(tmp_path / "element.txt", e, fmt="%d")
    return T.read_mesh_dir(str(tmp_path), 8, 1)


def test_reference_bc_files_through_the_reader(T, tmp_path):
    """InputMeshData::GetBcs (InputMeshData.cpp:228-285) reads Load = 41 load
    DOFs and values and StrucDofs = 8733 fixed DOFs (OptPara.cpp:5-11); the
    library's reader returns exactly the files' numbers: whole nodes clamped
    (DOF triples 3n, 3n+1, 3n+2) and unit loads on y DOFs (3n+1)."""
    _, _, f, ld, lv, cp = read_reference_bcs(T, tmp_path)
    assert f.size == 8733 and ld.size == 41 and lv.size == 41 and list(cp) == [0, 41]
    raw = lambda n: np.loadtxt(os.path.join(REF_MESH, n)).ravel()
    assert np.array_equal(f, raw("fixeddofs.txt").astype(np.int32))
    assert np.array_equal(ld, raw("loaddof_1.txt").astype(np.int32))
    assert np.array_equal(lv, raw("load_1.txt"))
    trip = f.reshape(-1, 3)
    assert np.all(trip[:, 0] % 3 == 0) and np.all(trip == trip[:, :1] + np.arange(3))
    assert np.all(ld % 3 == 1) and np.all(lv == 1.0)
    assert np.unique(f).size == f.size and np.unique(ld).size == ld.size
    ref = os.environ.get("TOPO_REFERENCE_ROOT")  # where a checkout of the reference is at hand
    if ref and os.path.isdir(os.path.join(ref, "mesh")):
        for name in ("fixeddofs.txt", "loaddof_1.txt", "load_1.txt"):
            with open(os.path.join(ref, "mesh", name), "rb") as a, open(os.path.join(REF_MESH, name), "rb") as b:
                assert a.read() == b.read(), name


def _create(T, v, e, f, ld, lv, **kw):
    return T.Context(v, e, f, ld, lv, stream=0, **kw)


def test_invalid_mesh_rejected_before_any_device_work(T):
    v, e, f, ld, lv = T.gen_cantilever(3, 2, 2, 8)
    bad = e.copy()
    bad[1, 3] = v.shape[0] + 5
    with pytest.raises(T.TopoError) as ei:
        _create(T, v, bad, f, ld, lv)
    assert ei.value.code == -4 and "outside" in str(ei.value)
    vn = v.copy()
    vn[2, 1] = np.nan
    with pytest.raises(T.TopoError) as ei:
        _create(T, vn, e, f, ld, lv)
    assert ei.value.code == -4 and "not finite" in str(ei.value)
    with pytest.raises(T.TopoError) as ei:
        _create(T, v, e, f, ld, lv * np.nan)
    assert ei.value.code == -4
    with pytest.raises(T.TopoError) as ei:
        _create(T, v, e, f, ld, lv, m=9)
    assert ei.value.code == -1


def test_driver_program_fails_loudly_without_a_gpu(tmp_path):
    """The main.cpp-shaped driver (`topopt`, over include/topopt.hpp) has no
    CPU fallback: without a CUDA device it stops at topo_create with the
    library's error and a nonzero status.  On a GPU machine it must run a
    tiny lattice to the end instead."""
    import subprocess
    import torch
    exe = os.path.join(ROOT, "unstructured-fea-based-topology-optimization-in-petsc-and-eigen_b200", "topopt")
    assert os.path.exists(exe)
    r = subprocess.run([exe, "-lattice", "4", "2", "2", "-maxItr", "2"], cwd=tmp_path, capture_output=True,
                       text=True, timeout=120)
    if torch.cuda.is_available():
        assert r.returncode == 0, r.stderr
    else:
        assert r.returncode != 0
        assert "no CPU fallback" in r.stderr


@pytest.mark.parametrize("field,value", [("cheb_degree_coarse", 16), ("cheb_degree_post", -1), ("amg_max_levels", 0),
                                         ("amg_max_levels", 9), ("amg_rho_its", -2), ("cheb_safety", -0.5),
                                         ("pdl", 2), ("fem_graphs", -1), ("autotune", 3), ("amg_half_fine", 2),
                                         ("fem_block", 5), ("proj", 2), ("amg_coarse_max", 5), ("cheb_degree", 0),
                                         ("step_graph", 2), ("blk_stages", 1), ("blk_stages", 4),
                                         ("deterministic", 2)])
def test_invalid_solver_options_rejected_before_any_device_work(T, field, value):
    """Out-of-range solver options are refused at creation with the option's
    name in the message (no silent clamping), before any device call."""
    v, e, f, ld, lv = T.gen_cantilever(3, 2, 2, 8)
    with pytest.raises(T.TopoError) as ei:
        _create(T, v, e, f, ld, lv, **{field: value})
    assert ei.value.code == -1 and field in str(ei.value)


def test_job_footprint_estimate_is_monotone(T):
    """The serving admission estimate grows with the mesh, is larger for the
    FP64 form than for the mixed one, and covers the per-element node-row Ke
    copy of the level-0 assembly (3 x 3nen values per (element, node) pair)."""
    for nen in (8, 4):
        small = T.estimate_job_bytes(nen, 10_000, 9_000, T.PREC_MIXED)
        big = T.estimate_job_bytes(nen, 400_000, 390_000, T.PREC_MIXED)
        assert big > small > 96 * (1 << 20)
        assert T.estimate_job_bytes(nen, 400_000, 390_000, T.PREC_FP64) > big
        more_elems = T.estimate_job_bytes(nen, 400_000, 780_000, T.PREC_MIXED)
        assert more_elems - big >= 390_000 * 9 * nen * nen * 4


def test_batch_and_server_arguments_checked_on_the_host(T):
    """topo_opt_step_batch and the server's batching switch reject bad
    arguments before any device work."""
    import ctypes as C
    L = T.lib()
    assert L.topo_opt_step_batch(None, 1, None, None) == T.TOPO_ERR_ARG
    arr = (C.c_void_p * 2)(None, None)
    assert L.topo_opt_step_batch(arr, 2, None, None) == T.TOPO_ERR_ARG and "null context" in T.last_error()
    assert L.topo_opt_step_batch(arr, 0, None, None) == 0  # nothing to do
    assert L.topo_server_set_batching(None, 10) == T.TOPO_ERR_ARG


@pytest.mark.parametrize("nd", [24, 12])
def test_block_bank_layout_is_conflict_free(T, nd):
    """The block operator stores the packed element matrix permuted so that the
    distinct entries each half-warp reads for one m8n8k4 A fragment (lane l:
    row 8 mt + l/4, column 4 kt + l%4) sit at positions distinct mod 16, i.e.
    in distinct shared-memory banks for 64-bit loads.  Checked here against
    an independent restatement of the fragment layout (host only)."""
    import ctypes as C
    npk = nd * (nd + 1) // 2
    perm = (C.c_int32 * npk)()
    assert T.lib().topo_test_block_bank_layout(nd, perm) == 1
    p = np.array(perm[:])
    assert sorted(p.tolist()) == list(range(npk))

    def pk(i, j):
        i, j = min(i, j), max(i, j)
        return i * nd - i * (i - 1) // 2 + (j - i)

    for mt in range((nd + 7) // 8):
        for kt in range((nd + 3) // 4):
            for half in range(2):
                ks = {pk(8 * mt + l // 4, 4 * kt + l % 4) for l in range(16 * half, 16 * half + 16)
                      if 8 * mt + l // 4 < nd}
                res = [p[k] % 16 for k in ks]
                assert len(set(res)) == len(res), (mt, kt, half)
    assert T.lib().topo_test_block_bank_layout(10, perm) == -1
