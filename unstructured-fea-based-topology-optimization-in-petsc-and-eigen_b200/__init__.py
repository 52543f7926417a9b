"""Python front end of libtopo.so, the sm_100a SIMP design-iteration library.

The library's product boundary is the C ABI in include/topo.h; this module
binds it with ctypes so that Python callers (tests, the benchmark, serving
drivers) can use it.  Device vectors are torch CUDA tensors (torch is used as
the device-memory and stream plumbing only).  The classes SolveFem, PDEFilter
and MMA mirror the reference's class interfaces (SolveFem.h, PDEFilter.h,
MMA.h) on top of one `Context` (one topology-optimisation job).

There is no CPU fallback: without a CUDA device every call that touches the
GPU raises TopoError.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtopo.so")

TOPO_OK = 0
TOPO_NOT_CONVERGED = 1
TOPO_ERR_ARG = -1
TOPO_ERR_NAN = -5
TOPO_ERR_TIMEOUT = -7
TOPO_ERR_CANCELLED = -9
PREC_FP64 = 0
PREC_MIXED = 1

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class Params(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "Emin", "Emax", "nu", "penal", "volfrac", "rmin", "Xmin", "Xmax", "movlim", "x0", "beta0", "betamax")] + [
        ("proj", C.c_int), ("maxItr", C.c_int), ("m", C.c_int), ("ch_tol", C.c_double),
        ("fem_rtol", C.c_double), ("fem_restart", C.c_int), ("fem_maxit", C.c_int), ("precision", C.c_int),
        ("amg_max_levels", C.c_int), ("amg_coarse_max", C.c_int), ("amg_smooth_p", C.c_int),
        ("cheb_degree", C.c_int), ("fine_smoother_matfree", C.c_int),
        ("filter_rtol", C.c_double), ("filter_atol", C.c_double), ("filter_dtol", C.c_double),
        ("filter_maxit", C.c_int), ("verbose", C.c_int), ("amg_rho_its", C.c_int), ("cheb_safety", C.c_double),
        ("fem_warm_start", C.c_int),
        ("fem_block", C.c_int),
        ("fem_graphs", C.c_int),
        ("cheb_degree_post", C.c_int),
        ("cheb_degree_coarse", C.c_int),
        ("autotune", C.c_int),
        ("amg_coarse_cta", C.c_int),
        ("amg_half_fine", C.c_int),
        ("pdl", C.c_int),
        ("step_graph", C.c_int),
        ("blk_stages", C.c_int),
        ("deterministic", C.c_int)]


class SolveInfo(C.Structure):
    _fields_ = [("fem_its", C.c_int), ("fem_relres", C.c_double), ("fem_status", C.c_int),
                ("filter_its", C.c_int * 4), ("amg_levels", C.c_int), ("amg_dofs", C.c_int * 8),
                ("mma_inner_its", C.c_int), ("last_fx", C.c_double), ("last_gx0", C.c_double),
                ("last_ch", C.c_double), ("t_fem_ms", C.c_double), ("t_filter_ms", C.c_double),
                ("t_mma_ms", C.c_double), ("t_setup_ms", C.c_double), ("tuned", C.c_int * 4),
                ("tuned_lanes", C.c_int * 8), ("step_graph", C.c_int), ("t_capture_ms", C.c_double)]


class TopoError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


# every symbol include/topo.h declares, with its ctypes signature
_SIGS = {
    "topo_last_error": ([], C.c_char_p),
    "topo_version": ([], C.c_char_p),
    "topo_params_default": ([C.POINTER(Params)], None),
    "topo_struct_sizes": ([C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)], C.c_int),
    "topo_device_alloc": ([C.c_size_t, C.POINTER(C.c_void_p)], C.c_int),
    "topo_device_free": ([C.c_void_p], C.c_int),
    "topo_memcpy_h2d": ([C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p], C.c_int),
    "topo_memcpy_d2h": ([C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p], C.c_int),
    "topo_sync": ([C.c_void_p], C.c_int),
    "topo_create": ([C.POINTER(Params), C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                     C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p)], C.c_int),
    "topo_destroy": ([C.c_void_p], C.c_int),
    "topo_get_params": ([C.c_void_p, C.POINTER(Params)], C.c_int),
    "topo_set_params": ([C.c_void_p, C.POINTER(Params)], C.c_int),
    "topo_sizes": ([C.c_void_p] + [C.POINTER(C.c_int)] * 4, C.c_int),
    "topo_stream": ([C.c_void_p], C.c_void_p),
    "topo_fem_volumes": ([C.c_void_p, C.c_void_p, _dp], C.c_int),
    "topo_fem_element_matrix": ([C.c_void_p, C.c_int, C.c_void_p], C.c_int),
    "topo_fem_apply": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "topo_fem_apply_block": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "topo_fem_obj_sens": ([C.c_void_p, C.c_void_p, _dp, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "topo_fem_solve": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "topo_fem_displacement": ([C.c_void_p, C.c_void_p], C.c_int),
    "topo_fem_von_mises": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "topo_filter_apply": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_double], C.c_int),
    "topo_filter_sens": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_int], C.c_int),
    "topo_heaviside": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_int,
                        C.c_double, C.c_int], C.c_int),
    "topo_projected_sens": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_double], C.c_int),
    "topo_filter_state": ([C.c_void_p, C.c_void_p, C.c_int], C.c_int),
    "topo_mma_set_outer_movelimit": ([C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_void_p, C.c_void_p,
                                      C.c_void_p], C.c_int),
    "topo_mma_update": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
                        C.c_int),
    "topo_mma_design_change": ([C.c_void_p, C.c_void_p, C.c_void_p, _dp], C.c_int),
    "topo_mma_set_asymptotes": ([C.c_void_p, C.c_double, C.c_double, C.c_double], C.c_int),
    "topo_mma_set_robust_asymptotes_type": ([C.c_void_p, C.c_int], C.c_int),
    "topo_mma_constraint_modification": ([C.c_void_p, C.c_int], C.c_int),
    "topo_mma_restart": ([C.c_void_p] + [C.c_void_p] * 4 + [C.POINTER(C.c_int), C.c_int], C.c_int),
    "topo_mma_kkt_residual": ([C.c_void_p] + [C.c_void_p] * 6 + [_dp, _dp], C.c_int),
    "topo_opt_init": ([C.c_void_p], C.c_int),
    "topo_opt_step": ([C.c_void_p, C.POINTER(C.c_int), _dp, _dp, _dp], C.c_int),
    "topo_opt_run": ([C.c_void_p, C.c_int, C.c_void_p, C.POINTER(C.c_int)], C.c_int),
    "topo_opt_step_host": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, _dp], C.c_int),
    "topo_opt_step_batch": ([C.c_void_p, C.c_int, C.c_void_p, C.c_void_p], C.c_int),
    "topo_opt_step_async": ([C.c_void_p], C.c_int),
    "topo_opt_step_query": ([C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), _dp, _dp, _dp], C.c_int),
    "topo_fem_sensitivities_noalloc": ([C.c_int, C.c_int] + [C.c_void_p] * 5 + [C.c_double] * 5 +
                                       [C.c_void_p] * 4, C.c_int),
    "topo_estimate_job_bytes": ([C.c_int, C.c_int, C.c_int, C.c_int], C.c_size_t),
    "topo_server_create": ([C.c_size_t, C.c_int, C.POINTER(C.c_void_p)], C.c_int),
    "topo_server_destroy": ([C.c_void_p], C.c_int),
    "topo_server_submit": ([C.c_void_p, C.POINTER(Params), C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                            C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_double,
                            C.POINTER(C.c_int)], C.c_int),
    "topo_server_run": ([C.c_void_p], C.c_int),
    "topo_server_cancel": ([C.c_void_p, C.c_int], C.c_int),
    "topo_server_set_batching": ([C.c_void_p, C.c_int], C.c_int),
    "topo_test_wait_limits": ([C.c_void_p, C.c_uint, C.c_ulonglong, C.c_int], C.c_int),
    "topo_test_block_bank_layout": ([C.c_int, C.POINTER(C.c_int32)], C.c_int),
    "topo_server_job": ([C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)] + [C.c_void_p] * 3 +
                        [_dp, _dp], C.c_int),
    "topo_server_stats_get": ([C.c_void_p, C.c_void_p], C.c_int),
    "topo_kernel_launches": ([], C.c_long),
    "topo_profile_enable": ([C.c_void_p, C.c_int], C.c_int),
    "topo_profile_read": ([C.c_void_p, C.c_int, C.POINTER(C.c_long), _dp], C.c_int),
    "topo_graph_aggregate": ([C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "topo_amg_level": ([C.c_void_p, C.c_int, C.c_int] + [C.POINTER(C.c_int)] * 4 + [C.POINTER(C.c_long)] +
                       [C.c_void_p] * 3, C.c_int),
    "topo_opt_vector": ([C.c_void_p, C.c_int, C.POINTER(C.c_void_p)], C.c_int),
    "topo_solve_info_get": ([C.c_void_p, C.POINTER(SolveInfo)], C.c_int),
    "topo_gen_cantilever": ([C.c_int] * 4 + [C.c_double, C.c_uint64, C.c_int] + [C.c_void_p] * 5 +
                            [C.POINTER(C.c_int)] * 4, C.c_int),
    "topo_gen_multiload": ([C.c_int] * 4 + [C.c_uint64, C.c_void_p, C.c_void_p], C.c_int),
    "topo_read_mesh_dir": ([C.c_char_p, C.c_int, C.c_int] + [C.c_void_p] * 6 + [C.POINTER(C.c_int)] * 4, C.c_int),
    "topo_write_vtu": ([C.c_void_p, C.c_char_p, C.c_int, C.c_void_p], C.c_int),
}

_lib = None


def lib():
    """Load libtopo.so (built in-tree by build.py) and bind every symbol."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise TopoError(-2, f"{LIB_PATH} is missing: run build.py (there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def symbols():
    return list(_SIGS)


def kernel_launches() -> int:
    return lib().topo_kernel_launches()


def graph_aggregate(rp, ci, excl=None):
    """Greedy aggregation of a node graph (host; same routine the AMG uses)."""
    rp = np.ascontiguousarray(rp, dtype=np.int32)
    ci = np.ascontiguousarray(ci, dtype=np.int32)
    n = rp.size - 1
    agg = np.zeros(n, dtype=np.int32)
    ex = None if excl is None else np.ascontiguousarray(excl, dtype=np.uint8)
    na = _check(lib().topo_graph_aggregate(n, _ptr(rp), _ptr(ci), None if ex is None else _ptr(ex), _ptr(agg)),
                "graph_aggregate")
    return na, agg


def last_error() -> str:
    return lib().topo_last_error().decode()


def _check(rc, what):
    if rc < 0:
        raise TopoError(rc, f"{what}: {last_error()}")
    return rc


def default_params(**kw) -> Params:
    p = Params()
    lib().topo_params_default(C.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise AttributeError(k)
        setattr(p, k, v)
    return p


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


# ---------------------------------------------------------------- meshes
def gen_cantilever(nx, ny, nz, nen=8, jitter=None, seed=2024, load_mode=0):
    """Seeded jittered cantilever lattice (host arrays)."""
    if jitter is None:
        jitter = 0.1 if nen == 8 else 0.2
    nn, ne, nf, nl = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    L = lib()
    _check(L.topo_gen_cantilever(nx, ny, nz, nen, jitter, seed, load_mode, None, None, None, None, None,
                                 C.byref(nn), C.byref(ne), C.byref(nf), C.byref(nl)), "gen_cantilever")
    v = np.zeros(nn.value * 3)
    e = np.zeros(ne.value * nen, dtype=np.int32)
    f = np.zeros(nf.value, dtype=np.int32)
    ld = np.zeros(nl.value, dtype=np.int32)
    lv = np.zeros(nl.value)
    _check(L.topo_gen_cantilever(nx, ny, nz, nen, jitter, seed, load_mode, _ptr(v), _ptr(e), _ptr(f), _ptr(ld),
                                 _ptr(lv), C.byref(nn), C.byref(ne), C.byref(nf), C.byref(nl)), "gen_cantilever")
    return v.reshape(-1, 3), e.reshape(-1, nen), f, ld, lv


def gen_multiload(nx, ny, nz, k, seed=2025):
    ld = np.zeros(3 * k, dtype=np.int32)
    lv = np.zeros(3 * k)
    _check(lib().topo_gen_multiload(nx, ny, nz, k, seed, _ptr(ld), _ptr(lv)), "gen_multiload")
    return ld, lv


def read_mesh_dir(path, nen=8, n_cases=1):
    nn, ne, nf, nl = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    L = lib()
    b = path.encode()
    _check(L.topo_read_mesh_dir(b, nen, n_cases, None, None, None, None, None, None, C.byref(nn), C.byref(ne),
                                C.byref(nf), C.byref(nl)), "read_mesh_dir")
    v = np.zeros(nn.value * 3)
    e = np.zeros(ne.value * nen, dtype=np.int32)
    f = np.zeros(nf.value, dtype=np.int32)
    cp = np.zeros(n_cases + 1, dtype=np.int32)
    ld = np.zeros(nl.value, dtype=np.int32)
    lv = np.zeros(nl.value)
    _check(L.topo_read_mesh_dir(b, nen, n_cases, _ptr(v), _ptr(e), _ptr(f), _ptr(cp), _ptr(ld), _ptr(lv),
                                C.byref(nn), C.byref(ne), C.byref(nf), C.byref(nl)), "read_mesh_dir")
    return v.reshape(-1, 3), e.reshape(-1, nen), f, ld, lv, cp


# ---------------------------------------------------------------- context
def _torch():
    import torch
    return torch


def _dptr(t):
    if t is None:
        return None
    assert t.is_cuda and t.is_contiguous(), "device tensors must be contiguous CUDA tensors"
    return C.c_void_p(t.data_ptr())


class Context:
    """One job: device-resident mesh + SolveFem + PDEFilter + MMA state."""

    def __init__(self, vertex, element, fixed, load_dofs, load_vals, case_ptr=None, params: Optional[Params] = None,
                 stream=None, **kw):
        torch = _torch()
        self.params = params if params is not None else default_params(**kw)
        vertex = np.ascontiguousarray(vertex, dtype=np.float64).reshape(-1)
        element = np.ascontiguousarray(element, dtype=np.int32)
        nen = element.shape[1] if element.ndim == 2 else 8
        fixed = np.ascontiguousarray(fixed, dtype=np.int32)
        ld = np.ascontiguousarray(load_dofs, dtype=np.int32)
        lv = np.ascontiguousarray(load_vals, dtype=np.float64)
        if case_ptr is None:
            case_ptr = np.array([0, ld.size], dtype=np.int32)
        case_ptr = np.ascontiguousarray(case_ptr, dtype=np.int32)
        self.nen, self.nn, self.ne = nen, vertex.size // 3, element.size // nen
        self.ndof, self.ncases = 3 * self.nn, case_ptr.size - 1
        if stream is None:
            # torch's current stream; its legacy default stream (handle 0) is
            # passed as cudaStreamLegacy (1) so that the library's work stays
            # ordered with torch's instead of getting a stream of its own
            stream = torch.cuda.current_stream().cuda_stream or 1
        elif stream == "own":
            stream = 0  # the library creates a stream for this context
        self.stream = stream
        h = C.c_void_p()
        _check(lib().topo_create(C.byref(self.params), nen, self.nn, _ptr(vertex), self.ne, _ptr(element.reshape(-1)),
                                 fixed.size, _ptr(fixed), self.ncases, _ptr(case_ptr), _ptr(ld), _ptr(lv),
                                 C.c_void_p(stream), C.byref(h)), "topo_create")
        self.h = h
        self.m = self.params.m

    def close(self):
        if getattr(self, "h", None):
            lib().topo_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---------------- helpers
    def zeros(self, n):
        torch = _torch()
        return torch.zeros(n, dtype=torch.float64, device="cuda")

    def set_params(self, **kw):
        for k, v in kw.items():
            setattr(self.params, k, v)
        _check(lib().topo_set_params(self.h, C.byref(self.params)), "topo_set_params")

    def info(self) -> SolveInfo:
        s = SolveInfo()
        _check(lib().topo_solve_info_get(self.h, C.byref(s)), "info")
        return s

    # ---------------- SolveFem
    def volumes(self):
        vol = self.zeros(self.ne)
        tv = C.c_double()
        _check(lib().topo_fem_volumes(self.h, _dptr(vol), C.byref(tv)), "volumes")
        return vol, tv.value

    def element_matrix(self, e):
        nd = 3 * self.nen
        k = np.zeros(nd * nd)
        _check(lib().topo_fem_element_matrix(self.h, e, _ptr(k)), "element_matrix")
        return k.reshape(nd, nd)

    def fem_apply(self, xphys, u):
        y = self.zeros(self.ndof)
        _check(lib().topo_fem_apply(self.h, _dptr(xphys), _dptr(u), _dptr(y)), "fem_apply")
        return y

    def fem_apply_block(self, xphys, u):
        """K(xphys) applied to every load case at once; u is [n_cases][ndof]."""
        y = self.zeros(self.ncases * self.ndof)
        _check(lib().topo_fem_apply_block(self.h, _dptr(xphys), _dptr(u), _dptr(y)), "fem_apply_block")
        return y

    def fem_obj_sens(self, xphys):
        fx = C.c_double()
        gx = np.zeros(self.m)
        df = self.zeros(self.ne)
        dg = self.zeros(self.ne * self.m)
        rc = _check(lib().topo_fem_obj_sens(self.h, _dptr(xphys), C.byref(fx), gx.ctypes.data_as(_dp), _dptr(df),
                                            _dptr(dg)), "fem_obj_sens")
        return fx.value, gx, df, dg.view(self.m, self.ne), rc

    def fem_solve(self, xphys):
        U = self.zeros(self.ndof * self.ncases)
        rc = _check(lib().topo_fem_solve(self.h, _dptr(xphys), _dptr(U)), "fem_solve")
        return U, rc

    def displacement(self):
        U = self.zeros(self.ndof * self.ncases)
        _check(lib().topo_fem_displacement(self.h, _dptr(U)), "displacement")
        return U

    def von_mises(self, xphys):
        v = self.zeros(self.ne)
        _check(lib().topo_fem_von_mises(self.h, _dptr(xphys), _dptr(v)), "von_mises")
        return v

    # ---------------- PDEFilter
    def filter(self, x, Xmin=None):
        xf = self.zeros(self.ne)
        rc = _check(lib().topo_filter_apply(self.h, _dptr(x), _dptr(xf), self.params.Xmin if Xmin is None else Xmin),
                    "filter")
        return xf

    def filter_sens(self, dfdx, dgdx):
        df = dfdx.clone().contiguous()
        dg = dgdx.clone().contiguous()
        m = dg.numel() // self.ne
        _check(lib().topo_filter_sens(self.h, _dptr(df), _dptr(dg), m), "filter_sens")
        return df, dg.view(m, self.ne)

    def filter_state(self, rx=None):
        if rx is None:
            out = self.zeros(self.nn)
            _check(lib().topo_filter_state(self.h, _dptr(out), 0), "filter_state")
            return out
        _check(lib().topo_filter_state(self.h, _dptr(rx.contiguous()), 1), "filter_state")

    def heaviside(self, xf, itr, x0=0.5, beta0=1.0, betamax=8.0, Xmin=0.01, proj=0):
        xp = self.zeros(self.ne)
        _check(lib().topo_heaviside(self.h, _dptr(xf), _dptr(xp), x0, beta0, betamax, itr, Xmin, proj), "heaviside")
        return xp

    def projected_sens(self, xf, dfdx, dgdx, x0=0.5):
        df = dfdx.clone().contiguous()
        dg = dgdx.clone().contiguous()
        m = dg.numel() // self.ne
        _check(lib().topo_projected_sens(self.h, _dptr(xf), _dptr(df), _dptr(dg), m, x0), "projected_sens")
        return df, dg.view(m, self.ne)

    # ---------------- MMA
    def mma_movelimit(self, x, Xmin=0.01, Xmax=1.0, movlim=0.2):
        a, b = self.zeros(self.ne), self.zeros(self.ne)
        _check(lib().topo_mma_set_outer_movelimit(self.h, Xmin, Xmax, movlim, _dptr(x), _dptr(a), _dptr(b)),
               "movelimit")
        return a, b

    def mma_update(self, x, dfdx, gx, dgdx, xmin, xmax):
        xv = x.clone().contiguous()
        g = np.ascontiguousarray(gx, dtype=np.float64)
        _check(lib().topo_mma_update(self.h, _dptr(xv), _dptr(dfdx.contiguous()), _ptr(g),
                                     _dptr(dgdx.contiguous()), _dptr(xmin), _dptr(xmax)), "mma_update")
        return xv

    def mma_design_change(self, x, xold):
        xo = xold.clone().contiguous()
        ch = C.c_double()
        _check(lib().topo_mma_design_change(self.h, _dptr(x), _dptr(xo), C.byref(ch)), "design_change")
        return ch.value, xo

    def mma_state(self):
        """(xo1, xo2, L, U, k) of the MMA history (MMA::Restart order is xo1, xo2, U, L)."""
        xo1, xo2, L, U = [self.zeros(self.ne) for _ in range(4)]
        k = C.c_int()
        _check(lib().topo_mma_restart(self.h, _dptr(xo1), _dptr(xo2), _dptr(U), _dptr(L), C.byref(k), 0),
               "mma_restart")
        return [xo1, xo2, L, U, k.value]

    def mma_options(self, asyminit=0.5, asymdec=0.7, asyminc=1.2, robust=0, constraint_mod=0):
        """MMA::SetAsymptotes, SetRobustAsymptotesType and the
        constraintModification flag."""
        L = lib()
        _check(L.topo_mma_set_asymptotes(self.h, asyminit, asymdec, asyminc), "mma_set_asymptotes")
        _check(L.topo_mma_set_robust_asymptotes_type(self.h, robust), "mma_set_robust_asymptotes_type")
        _check(L.topo_mma_constraint_modification(self.h, constraint_mod), "mma_constraint_modification")

    def mma_restart_set(self, xo1, xo2, U, L, k):
        """The restart constructor's import of the MMA history (MMA.h:15-18)."""
        kk = C.c_int(k)
        _check(lib().topo_mma_restart(self.h, _dptr(xo1.contiguous()), _dptr(xo2.contiguous()),
                                      _dptr(U.contiguous()), _dptr(L.contiguous()), C.byref(kk), 1), "mma_restart")

    def mma_kkt(self, x, dfdx, gx, dgdx, xmin, xmax):
        n2, ni = C.c_double(), C.c_double()
        g = np.ascontiguousarray(gx, dtype=np.float64)
        _check(lib().topo_mma_kkt_residual(self.h, _dptr(x), _dptr(dfdx), _ptr(g), _dptr(dgdx), _dptr(xmin),
                                           _dptr(xmax), C.byref(n2), C.byref(ni)), "kkt")
        return n2.value, ni.value

    # ---------------- main loop
    def opt_init(self):
        _check(lib().topo_opt_init(self.h), "opt_init")

    def opt_step(self):
        it, fx, gx, ch = C.c_int(), C.c_double(), C.c_double(), C.c_double()
        rc = _check(lib().topo_opt_step(self.h, C.byref(it), C.byref(fx), C.byref(gx), C.byref(ch)), "opt_step")
        return it.value, fx.value, gx.value, ch.value

    def opt_step_async(self):
        """Start one design iteration without waiting for it."""
        _check(lib().topo_opt_step_async(self.h), "opt_step_async")

    def opt_step_query(self):
        """None while the started iteration runs, else (status, itr, fx, gx0, ch)."""
        done, it, fx, gx, ch = C.c_int(), C.c_int(), C.c_double(), C.c_double(), C.c_double()
        rc = _check(lib().topo_opt_step_query(self.h, C.byref(done), C.byref(it), C.byref(fx), C.byref(gx),
                                              C.byref(ch)), "opt_step_query")
        return (rc, it.value, fx.value, gx.value, ch.value) if done.value else None

    def opt_run(self, max_itr):
        hist = np.zeros(3 * max_itr)
        n = C.c_int()
        _check(lib().topo_opt_run(self.h, max_itr, _ptr(hist), C.byref(n)), "opt_run")
        return hist.reshape(-1, 3)[:n.value]

    def opt_step_host(self, x_in: np.ndarray, x_out: np.ndarray, xphys_out: np.ndarray):
        """One design iteration with host buffers (x_in -> x_out, xphys_out)."""
        fx = C.c_double()
        _check(lib().topo_opt_step_host(self.h, _ptr(x_in), _ptr(x_out), _ptr(xphys_out), C.byref(fx)),
               "opt_step_host")
        return fx.value

    def amg_level(self, level, which):
        """Level matrix as a scipy BSR/CSR matrix (which: 0 A, 1 P, 2 R)."""
        import scipy.sparse as sp
        nr, nc, br, bc, nb = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_long()
        L = lib()
        _check(L.topo_amg_level(self.h, level, which, C.byref(nr), C.byref(nc), C.byref(br), C.byref(bc),
                                C.byref(nb), None, None, None), "amg_level")
        rp = np.zeros(nr.value + 1, dtype=np.int32)
        ci = np.zeros(nb.value, dtype=np.int32)
        vals = np.zeros(nb.value * br.value * bc.value)
        _check(L.topo_amg_level(self.h, level, which, C.byref(nr), C.byref(nc), C.byref(br), C.byref(bc),
                                C.byref(nb), _ptr(rp), _ptr(ci), _ptr(vals)), "amg_level")
        m = sp.bsr_matrix((vals.reshape(-1, br.value, bc.value), ci, rp),
                          shape=(nr.value * br.value, nc.value * bc.value))
        return m.tocsr()

    def profile(self, on=True):
        _check(lib().topo_profile_enable(self.h, 1 if on else 0), "profile_enable")

    def profile_read(self, slot):
        n, ms = C.c_long(), C.c_double()
        _check(lib().topo_profile_read(self.h, slot, C.byref(n), C.byref(ms)), "profile_read")
        return n.value, ms.value

    def opt_vector(self, which):
        """Device pointer (int) of one of the context's design vectors."""
        p = C.c_void_p()
        _check(lib().topo_opt_vector(self.h, which, C.byref(p)), "opt_vector")
        return p.value

    def opt_tensor(self, which, n=None):
        """Copy of a context design vector (0 X, 1 XPhys, 2 XFiled, 3 Xold,
        4 dfdx, 5 dgdx, 6 xmin, 7 xmax) as a torch tensor."""
        n = n or (self.ne * self.m if which == 5 else self.ne)
        return device_view(self.opt_vector(which), n).clone()

    def test_wait_limits(self, barrier_spins=0, copy_cycles=0, hold=0):
        """Bounds of the device-side waits; hold=1 makes them run out (tests of
        the timeout path)."""
        _check(lib().topo_test_wait_limits(self.h, barrier_spins, copy_cycles, hold), "test_wait_limits")

    def write_vtu(self, directory, itr, xphys=None):
        _check(lib().topo_write_vtu(self.h, directory.encode(), itr, _dptr(xphys)), "write_vtu")


def opt_step_batch(contexts):
    """One design iteration of every context at once (topo_opt_step_batch):
    returns (statuses, compliances).  Errors are reported per instance in the
    statuses, not raised."""
    n = len(contexts)
    arr = (C.c_void_p * max(n, 1))(*[c.h for c in contexts])
    st = np.zeros(max(n, 1), dtype=np.int32)
    fx = np.zeros(max(n, 1))
    lib().topo_opt_step_batch(arr, n, _ptr(st), _ptr(fx))
    return st[:n], fx[:n]


def device_view(ptr, n):
    """Zero-copy torch view of n doubles at a device pointer."""
    torch = _torch()

    class _Arr:
        __cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 3}

    return torch.as_tensor(_Arr(), device="cuda")


# ---------------------------------------------------------------- serving
class ServerStats(C.Structure):
    _fields_ = [("jobs_submitted", C.c_int), ("jobs_done", C.c_int), ("jobs_failed", C.c_int),
                ("max_active", C.c_int), ("iterations", C.c_long), ("p50_iter_ms", C.c_double),
                ("p99_iter_ms", C.c_double), ("mean_iter_ms", C.c_double), ("makespan_s", C.c_double),
                ("jobs_per_hour", C.c_double), ("iters_per_s", C.c_double), ("peak_reserved_bytes", C.c_double),
                ("p50_queue_s", C.c_double), ("p99_queue_s", C.c_double)]


def estimate_job_bytes(nen, n_nodes, n_elems, precision=PREC_FP64):
    return lib().topo_estimate_job_bytes(nen, n_nodes, n_elems, precision)


class Server:
    """Continuous-batching job server (topo_server_*)."""

    def __init__(self, hbm_budget_bytes=0, max_active=8, batch_max_elems=0):
        h = C.c_void_p()
        _check(lib().topo_server_create(hbm_budget_bytes, max_active, C.byref(h)), "server_create")
        self.h = h
        self.jobs = []
        if batch_max_elems:
            _check(lib().topo_server_set_batching(h, batch_max_elems), "server_set_batching")

    def submit(self, vertex, element, fixed, load_dofs, load_vals, iterations, arrival_s=0.0, case_ptr=None,
               params=None, **kw):
        p = params if params is not None else default_params(**kw)
        vertex = np.ascontiguousarray(vertex, dtype=np.float64).reshape(-1)
        element = np.ascontiguousarray(element, dtype=np.int32)
        nen = element.shape[1]
        fixed = np.ascontiguousarray(fixed, dtype=np.int32)
        ld = np.ascontiguousarray(load_dofs, dtype=np.int32)
        lv = np.ascontiguousarray(load_vals, dtype=np.float64)
        cp = np.ascontiguousarray(case_ptr if case_ptr is not None else [0, ld.size], dtype=np.int32)
        jid = C.c_int()
        _check(lib().topo_server_submit(self.h, C.byref(p), nen, vertex.size // 3, _ptr(vertex), element.shape[0],
                                        _ptr(element.reshape(-1)), fixed.size, _ptr(fixed), cp.size - 1, _ptr(cp),
                                        _ptr(ld), _ptr(lv), iterations, arrival_s, C.byref(jid)), "server_submit")
        self.jobs.append((jid.value, element.shape[0], iterations))
        return jid.value

    def run(self):
        return _check(lib().topo_server_run(self.h), "server_run")

    def cancel(self, jid):
        """Cancel a job (safe while run() is blocking in another thread)."""
        _check(lib().topo_server_cancel(self.h, jid), "server_cancel")

    def job(self, jid):
        _, ne, iters = self.jobs[jid]
        st, n = C.c_int(), C.c_int()
        lat = np.zeros(iters)
        fx = np.zeros(iters)
        xp = np.zeros(ne)
        a, f = C.c_double(), C.c_double()
        rc = lib().topo_server_job(self.h, jid, C.byref(st), C.byref(n), _ptr(lat), _ptr(fx), _ptr(xp), C.byref(a),
                                   C.byref(f))
        return dict(rc=rc, status=st.value, iter_ms=lat[:n.value], fx=fx[:n.value], xphys=xp, admit_s=a.value,
                    finish_s=f.value)

    def stats(self):
        s = ServerStats()
        _check(lib().topo_server_stats_get(self.h, C.byref(s)), "server_stats")
        return {k: getattr(s, k) for k, _ in ServerStats._fields_}

    def close(self):
        if getattr(self, "h", None):
            lib().topo_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- reference-shaped classes
class SolveFem:
    """SolveFem (SolveFem.h:12-55) over a Context."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        self.Vol, self.TV = ctx.volumes()

    def ComputeObjectiveAndSensitivities(self, XPhys):
        fx, gx, df, dg, _ = self.ctx.fem_obj_sens(XPhys)
        return fx, gx, df, dg

    @property
    def U(self):
        return self.ctx.displacement()


class PDEFilter:
    """PDEFilter (PDEFilter.h:12-56) over a Context."""

    def __init__(self, ctx: Context):
        self.ctx = ctx

    def Filter(self, X, Xmin):
        return self.ctx.filter(X, Xmin)

    def ComputeFilteredSens(self, dfdx, dgdx):
        return self.ctx.filter_sens(dfdx, dgdx)

    def HeavisideFilter(self, XFiled, x0, beta0, betamax, itr, Xmin, proj):
        return self.ctx.heaviside(XFiled, itr, x0, beta0, betamax, Xmin, proj)

    def ComputeProjectedSens(self, XFiled, dfdx, dgdx, x0):
        return self.ctx.projected_sens(XFiled, dfdx, dgdx, x0)


class MMA:
    """MMA (MMA.h:8-119) over a Context (a = 0, c = 1000, d = 0)."""

    def __init__(self, ctx: Context):
        self.ctx = ctx

    def SetOuterMovelimit(self, Xmin, Xmax, movlim, x):
        return self.ctx.mma_movelimit(x, Xmin, Xmax, movlim)

    def Update(self, xval, dfdx, gx, dgdx, xmin, xmax):
        return self.ctx.mma_update(xval, dfdx, gx, dgdx, xmin, xmax)

    def DesignChange(self, x, xold):
        return self.ctx.mma_design_change(x, xold)
