"""Outputs beside the design iteration, through the C ABI: the von Mises
stress per element (stress/ComputeStress.cpp:53-104) against the oracle's
restatement, and the VTU writer (Write2Vtu.cpp:5-174): counts, the
diagonal -> VTK node order, cell types, and the written fields.

Tolerances: von Mises 1e-10 relative (FP64, summation order only); VTU
values as printed (%e, 7 significant digits)."""
import xml.etree.ElementTree as ET

import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

KW = dict(Emax=1.0, rmin=1.5, volfrac=0.12, fem_rtol=1e-10)


def dev(cuda, a):
    return cuda.tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")


def test_von_mises_matches_oracle(T, O, cuda):
    v, e, f, ld, lv = T.gen_cantilever(10, 5, 4, 8)
    ctx = T.Context(v, e, f, ld, lv, **KW)
    x = np.random.default_rng(8).uniform(0.05, 1.0, e.shape[0])
    xd = dev(cuda, x)
    ctx.fem_obj_sens(xd)
    U = ctx.displacement().cpu().numpy()
    vm = ctx.von_mises(xd).cpu().numpy()
    p = ctx.params
    ref = []
    for el in range(e.shape[0]):
        nodes = e[el]
        ue = np.concatenate([U[3 * nodes + c] for c in range(3)])  # x0..x7, y0..y7, z0..z7
        ref.append(O.von_mises_hex8(v[nodes], p.nu, p.Emax, x[el], ue))
    assert rel(vm, np.array(ref)) < 1e-10
    assert np.all(vm >= 0)
    ctx.close()


@pytest.mark.parametrize("nen", [8, 4])
def test_vtu_writer(T, cuda, tmp_path, nen):
    dims = (6, 3, 2) if nen == 8 else (3, 2, 2)
    v, e, f, ld, lv = T.gen_cantilever(*dims, nen)
    ctx = T.Context(v, e, f, ld, lv, **KW)
    x = np.random.default_rng(2).uniform(0.1, 1.0, e.shape[0])
    xd = dev(cuda, x)
    ctx.fem_obj_sens(xd)
    U = ctx.displacement().cpu().numpy()
    ctx.write_vtu(str(tmp_path), 0, xd)
    ctx.write_vtu(str(tmp_path), 20, xd)
    ctx.write_vtu(str(tmp_path), -1, xd)
    for name in ("output_initial.vtu", "output_20.vtu", "output_final.vtu"):
        assert (tmp_path / name).exists()
    root = ET.parse(tmp_path / "output_initial.vtu").getroot()
    piece = root.find("UnstructuredGrid/Piece")
    assert int(piece.get("NumberOfPoints")) == v.shape[0] and int(piece.get("NumberOfCells")) == e.shape[0]
    arrays = {a.get("Name"): np.array(a.text.split(), dtype=float) for a in root.iter("DataArray")}
    assert np.allclose(arrays["nodes"].reshape(-1, 3), v, rtol=1e-6)
    conn = arrays["connectivity"].astype(int).reshape(-1, nen)
    order = [0, 1, 3, 2, 4, 5, 7, 6] if nen == 8 else [0, 1, 2, 3]  # diagonal -> VTK
    assert np.array_equal(conn, e[:, order])
    assert np.array_equal(arrays["offsets"].astype(int), nen * np.arange(1, e.shape[0] + 1))
    assert np.all(arrays["types"] == (12 if nen == 8 else 10))
    for c, nm in enumerate(("ux", "uy", "uz")):
        assert np.allclose(arrays[nm], U[c::3], rtol=1e-6, atol=1e-12 * np.abs(U).max())
    assert np.allclose(arrays["xphys"], x, rtol=1e-6)
    # an unwritable directory is an error, not an exit
    with pytest.raises(T.TopoError):
        ctx.write_vtu(str(tmp_path / "missing" / "dir"), 0, xd)
    ctx.close()
