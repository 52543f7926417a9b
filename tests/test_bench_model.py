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


def test_reference_arm_line_contract(tmp_path):
    """`bench.py --impl reference` (the CPU restatement timed on the host
    cores) prints one JSON line with the bench contract's keys, its own
    cpu_baseline and an e2e entry without host-device copies."""
    import json
    import os
    import subprocess
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "hex8-8k",
                        "--steps", "1", "--warmup", "0"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["workload"].startswith("hex8-8k")


def test_reference_arm_other_ranks_exit_quietly():
    """Under torchrun only rank 0 runs the reference arm; the other ranks exit
    0 without work or output."""
    import os
    import subprocess
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--workload", "hex8-8k", "--steps", "1", "--warmup", "0"], cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [l for l in r.stdout.splitlines() if l.startswith("{")]
