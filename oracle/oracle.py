"""ctypes front end of the CPU oracle (oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg.  The product never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
SRC = os.path.join(HERE, "oracle.c")

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def build(force: bool = False) -> str:
    """Compile oracle.c into liboracle.so (gcc, OpenMP)."""
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(
            os.path.getmtime(SRC), os.path.getmtime(os.path.join(HERE, "oracle.h"))):
        cmd = ["gcc", "-O3", "-fopenmp", "-fPIC", "-shared", "-o", LIB, SRC, "-lm"]
        subprocess.run(cmd, check=True)
    return LIB


class OrParams(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "Emin", "Emax", "nu", "penal", "volfrac", "rmin", "Xmin", "Xmax", "movlim", "x0", "beta0",
        "betamax")] + [("proj", C.c_int), ("maxItr", C.c_int), ("m", C.c_int),
                       ("fem_rtol", C.c_double), ("fem_restart", C.c_int), ("fem_maxit", C.c_int),
                       ("precond", C.c_int), ("amg_levels", C.c_int), ("amg_coarse_max", C.c_int),
                       ("cheb_degree", C.c_int), ("amg_smooth", C.c_int),
                       ("filter_rtol", C.c_double), ("filter_atol", C.c_double),
                       ("filter_dtol", C.c_double), ("filter_maxit", C.c_int), ("nthreads", C.c_int)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        L.or_gen_lattice_nodes.argtypes = [C.c_int] * 3 + [C.c_double, C.c_double, C.c_int, C.c_uint64, _f64p]
        L.or_gen_hex8_elements.argtypes = [C.c_int] * 3 + [_i32p]
        L.or_gen_tet4_elements.argtypes = [C.c_int] * 3 + [_f64p, _i32p]
        L.or_gen_tet4_elements.restype = C.c_int
        L.or_gen_cantilever_bcs.argtypes = [C.c_int] * 4 + [C.c_void_p] * 3 + [C.POINTER(C.c_int)] * 2
        L.or_gen_multiload.argtypes = [C.c_int] * 4 + [C.c_uint64, _i32p, _f64p]
        for nm, nd in (("or_hex8_ke", 24), ("or_tet4_ke", 12)):
            getattr(L, nm).argtypes = [_f64p, C.c_double, _f64p]
        L.or_hex8_volume.argtypes = [_f64p]
        L.or_hex8_volume.restype = C.c_double
        L.or_tet4_volume.argtypes = [_f64p]
        L.or_tet4_volume.restype = C.c_double
        L.or_hex8_kehel.argtypes = [_f64p, C.c_double, _f64p, _f64p]
        L.or_tet4_kehel.argtypes = [_f64p, C.c_double, _f64p, _f64p]
        L.or_von_mises_hex8.argtypes = [_f64p, C.c_double, C.c_double, C.c_double, _f64p, C.POINTER(C.c_double)]
        L.or_params_default.argtypes = [C.POINTER(OrParams)]
        L.or_create.argtypes = [C.POINTER(OrParams), C.c_int, C.c_int, _f64p, C.c_int, _i32p, C.c_int, _i32p,
                                C.c_int, _i32p, _i32p, _f64p]
        L.or_create.restype = C.c_void_p
        L.or_destroy.argtypes = [C.c_void_p]
        L.or_total_volume.argtypes = [C.c_void_p, C.c_void_p]
        L.or_total_volume.restype = C.c_double
        L.or_element_ke.argtypes = [C.c_void_p, C.c_int, _f64p]
        L.or_assemble.argtypes = [C.c_void_p, _f64p]
        L.or_get_csr.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                 C.POINTER(C.POINTER(C.c_int)), C.POINTER(C.POINTER(C.c_int)),
                                 C.POINTER(C.POINTER(C.c_double))]
        L.or_get_rhs.argtypes = [C.c_void_p, _f64p]
        L.or_kmatvec.argtypes = [C.c_void_p, _f64p, _f64p]
        L.or_solve.argtypes = [C.c_void_p, _f64p, C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.or_fem_obj_sens.argtypes = [C.c_void_p, _f64p, C.POINTER(C.c_double), _f64p, _f64p, _f64p, C.c_void_p]
        L.or_obj_sens_given_u.argtypes = [C.c_void_p, _f64p, _f64p, C.POINTER(C.c_double), _f64p, _f64p, _f64p]
        L.or_filter.argtypes = [C.c_void_p, _f64p, _f64p, C.c_double]
        L.or_filter_sens.argtypes = [C.c_void_p, _f64p, _f64p, C.c_int]
        L.or_filter_state.argtypes = [C.c_void_p, _f64p, C.c_int]
        L.or_filter_last_its.argtypes = [C.c_void_p]
        L.or_heaviside.argtypes = [C.c_void_p, _f64p, _f64p, C.c_double, C.c_double, C.c_double, C.c_int,
                                   C.c_double, C.c_int]
        L.or_projected_sens.argtypes = [C.c_void_p, _f64p, _f64p, _f64p, C.c_int, C.c_double]
        L.or_mma_set_outer_movelimit.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, _f64p, _f64p,
                                                 _f64p]
        L.or_mma_update.argtypes = [C.c_void_p, _f64p, _f64p, _f64p, _f64p, _f64p, _f64p]
        L.or_mma_design_change.argtypes = [C.c_void_p, _f64p, _f64p]
        L.or_mma_design_change.restype = C.c_double
        L.or_mma_state.argtypes = [C.c_void_p] + [C.c_void_p] * 4 + [C.POINTER(C.c_int)]
        L.or_mma_options.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int]
        L.or_mma_restart_set.argtypes = [C.c_void_p, _f64p, _f64p, _f64p, _f64p, C.c_int]
        L.or_mma_kkt_residual.argtypes = [C.c_void_p] + [_f64p] * 6 + [C.POINTER(C.c_double)] * 2
        L.or_amg_aggregates.argtypes = [C.c_void_p, C.c_int, _i32p]
        L.or_run.argtypes = [C.c_void_p, C.c_int, C.c_double, _f64p, _f64p]
        _lib = L
    return _lib


# ---------------------------------------------------------------- mesh
def lattice_nodes(nx, ny, nz, h=1.0, jitter=0.1, interior_only=False, seed=2024):
    v = np.zeros((nx + 1) * (ny + 1) * (nz + 1) * 3)
    lib().or_gen_lattice_nodes(nx, ny, nz, h, jitter, int(interior_only), seed, v)
    return v.reshape(-1, 3)


def hex8_elements(nx, ny, nz):
    e = np.zeros(nx * ny * nz * 8, dtype=np.int32)
    lib().or_gen_hex8_elements(nx, ny, nz, e)
    return e.reshape(-1, 8)


def tet4_elements(nx, ny, nz, vertex):
    e = np.zeros(nx * ny * nz * 24, dtype=np.int32)
    bad = lib().or_gen_tet4_elements(nx, ny, nz, np.ascontiguousarray(vertex, dtype=np.float64).ravel(), e)
    return e.reshape(-1, 4), bad


def cantilever_bcs(nx, ny, nz, load_mode=0):
    nf, nl = C.c_int(), C.c_int()
    lib().or_gen_cantilever_bcs(nx, ny, nz, load_mode, None, None, None, C.byref(nf), C.byref(nl))
    f = np.zeros(nf.value, dtype=np.int32)
    ld = np.zeros(nl.value, dtype=np.int32)
    lv = np.zeros(nl.value)
    lib().or_gen_cantilever_bcs(nx, ny, nz, load_mode, f.ctypes.data, ld.ctypes.data, lv.ctypes.data,
                                C.byref(nf), C.byref(nl))
    return f, ld, lv


def multiload(nx, ny, nz, k, seed=2025):
    ld = np.zeros(3 * k, dtype=np.int32)
    lv = np.zeros(3 * k)
    lib().or_gen_multiload(nx, ny, nz, k, seed, ld, lv)
    return ld, lv


def cantilever(nx, ny, nz, elem="hex8", seed=2024, jitter=None, load_mode=0):
    """Jittered cantilever box: (vertex, element, fixed, load_dofs, load_vals)."""
    if elem == "hex8":
        v = lattice_nodes(nx, ny, nz, 1.0, 0.1 if jitter is None else jitter, False, seed)
        e = hex8_elements(nx, ny, nz)
    else:
        v = lattice_nodes(nx, ny, nz, 1.0, 0.2 if jitter is None else jitter, True, seed)
        e, bad = tet4_elements(nx, ny, nz, v)
        assert bad == 0
    f, ld, lv = cantilever_bcs(nx, ny, nz, load_mode)
    return v, e, f, ld, lv


# ---------------------------------------------------------------- element level
def hex8_ke(co, nu=0.3):
    k = np.zeros(576)
    lib().or_hex8_ke(np.ascontiguousarray(co, dtype=np.float64).ravel(), nu, k)
    return k.reshape(24, 24)


def tet4_ke(co, nu=0.3):
    k = np.zeros(144)
    lib().or_tet4_ke(np.ascontiguousarray(co, dtype=np.float64).ravel(), nu, k)
    return k.reshape(12, 12)


def hex8_volume(co):
    return lib().or_hex8_volume(np.ascontiguousarray(co, dtype=np.float64).ravel())


def tet4_volume(co):
    return lib().or_tet4_volume(np.ascontiguousarray(co, dtype=np.float64).ravel())


def hex8_kehel(co, rmin):
    k, t = np.zeros(64), np.zeros(8)
    lib().or_hex8_kehel(np.ascontiguousarray(co, dtype=np.float64).ravel(), rmin, k, t)
    return k.reshape(8, 8), t


def tet4_kehel(co, rmin):
    k, t = np.zeros(16), np.zeros(4)
    lib().or_tet4_kehel(np.ascontiguousarray(co, dtype=np.float64).ravel(), rmin, k, t)
    return k.reshape(4, 4), t


def von_mises_hex8(co, nu, Emax, x, ue):
    out = C.c_double()
    lib().or_von_mises_hex8(np.ascontiguousarray(co, dtype=np.float64).ravel(), nu, Emax, x,
                            np.ascontiguousarray(ue, dtype=np.float64), C.byref(out))
    return out.value


# ---------------------------------------------------------------- system level
def default_params(**kw):
    p = OrParams()
    lib().or_params_default(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


class Oracle:
    """One CPU design-iteration context (mesh + SolveFem + PDEFilter + MMA)."""

    def __init__(self, vertex, element, fixed, load_dofs, load_vals, case_ptr=None, **params):
        self.p = default_params(**params)
        vertex = np.ascontiguousarray(vertex, dtype=np.float64).ravel()
        element = np.ascontiguousarray(element, dtype=np.int32)
        self.nen = element.shape[1]
        self.nn = vertex.size // 3
        self.ne = element.shape[0]
        self.n = 3 * self.nn
        ld = np.ascontiguousarray(load_dofs, dtype=np.int32)
        lv = np.ascontiguousarray(load_vals, dtype=np.float64)
        if case_ptr is None:
            case_ptr = np.array([0, ld.size], dtype=np.int32)
        case_ptr = np.ascontiguousarray(case_ptr, dtype=np.int32)
        self.ncases = case_ptr.size - 1
        self._keep = (vertex, element, fixed, ld, lv, case_ptr)
        self.h = lib().or_create(C.byref(self.p), self.nen, self.nn, vertex, self.ne, element.ravel(),
                                 len(fixed), np.ascontiguousarray(fixed, dtype=np.int32),
                                 self.ncases, case_ptr, ld, lv)
        if not self.h:
            raise ValueError("oracle: invalid mesh")

    def close(self):
        if self.h:
            lib().or_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def total_volume(self):
        vol = np.zeros(self.ne)
        tv = lib().or_total_volume(self.h, vol.ctypes.data)
        return tv, vol

    def element_ke(self, e):
        nd = 3 * self.nen
        k = np.zeros(nd * nd)
        lib().or_element_ke(self.h, e, k)
        return k.reshape(nd, nd)

    def assemble(self, xphys):
        lib().or_assemble(self.h, np.ascontiguousarray(xphys, dtype=np.float64))

    def csr(self):
        import scipy.sparse as sp
        n, nnz = C.c_int(), C.c_int()
        rp, ci, v = C.POINTER(C.c_int)(), C.POINTER(C.c_int)(), C.POINTER(C.c_double)()
        lib().or_get_csr(self.h, C.byref(n), C.byref(nnz), C.byref(rp), C.byref(ci), C.byref(v))
        rpa = np.ctypeslib.as_array(rp, (n.value + 1,)).copy()
        cia = np.ctypeslib.as_array(ci, (nnz.value,)).copy()
        va = np.ctypeslib.as_array(v, (nnz.value,)).copy()
        return sp.csr_matrix((va, cia, rpa), shape=(n.value, n.value))

    def rhs(self):
        F = np.zeros(self.n)
        lib().or_get_rhs(self.h, F)
        return F

    def kmatvec(self, u):
        y = np.zeros(self.n)
        lib().or_kmatvec(self.h, np.ascontiguousarray(u, dtype=np.float64), y)
        return y

    def solve(self):
        U = np.zeros(self.n)
        its, rr = C.c_int(), C.c_double()
        rc = lib().or_solve(self.h, U, C.byref(its), C.byref(rr))
        return U, its.value, rr.value, rc

    def fem_obj_sens(self, xphys, return_u=False):
        m = self.p.m
        fx = C.c_double()
        gx = np.zeros(m)
        df = np.zeros(self.ne)
        dg = np.zeros(self.ne * m)
        U = np.zeros(self.n)
        lib().or_fem_obj_sens(self.h, np.ascontiguousarray(xphys, dtype=np.float64), C.byref(fx), gx, df, dg,
                              U.ctypes.data)
        out = (fx.value, gx, df, dg.reshape(m, self.ne))
        return out + (U,) if return_u else out

    def obj_sens_given_u(self, xphys, U):
        """Compliance, volume constraint and sensitivities for a given U (no solve)."""
        m = self.p.m
        fx = C.c_double()
        gx = np.zeros(m)
        df = np.zeros(self.ne)
        dg = np.zeros(self.ne * m)
        lib().or_obj_sens_given_u(self.h, np.ascontiguousarray(xphys, dtype=np.float64),
                                  np.ascontiguousarray(U, dtype=np.float64), C.byref(fx), gx, df, dg)
        return fx.value, gx, df, dg.reshape(m, self.ne)

    def filter(self, x, Xmin):
        xf = np.zeros(self.ne)
        lib().or_filter(self.h, np.ascontiguousarray(x, dtype=np.float64), xf, Xmin)
        return xf

    def filter_sens(self, dfdx, dgdx):
        df = np.ascontiguousarray(dfdx, dtype=np.float64).copy()
        dg = np.ascontiguousarray(dgdx, dtype=np.float64).copy()
        m = dg.size // self.ne
        lib().or_filter_sens(self.h, df, dg.ravel(), m)
        return df, dg.reshape(m, self.ne)

    def filter_state(self, RX=None):
        if RX is None:
            out = np.zeros(self.nn)
            lib().or_filter_state(self.h, out, 0)
            return out
        lib().or_filter_state(self.h, np.ascontiguousarray(RX, dtype=np.float64), 1)

    def heaviside(self, xf, itr, x0=0.5, beta0=1.0, betamax=8.0, Xmin=0.01, proj=0):
        xp = np.zeros(self.ne)
        lib().or_heaviside(self.h, np.ascontiguousarray(xf, dtype=np.float64), xp, x0, beta0, betamax, itr,
                           Xmin, proj)
        return xp

    def projected_sens(self, xf, dfdx, dgdx, x0=0.5):
        df = np.ascontiguousarray(dfdx, dtype=np.float64).copy()
        dg = np.ascontiguousarray(dgdx, dtype=np.float64).copy()
        m = dg.size // self.ne
        lib().or_projected_sens(self.h, np.ascontiguousarray(xf, dtype=np.float64), df, dg.ravel(), m, x0)
        return df, dg.reshape(m, self.ne)

    def mma_movelimit(self, x, Xmin=0.01, Xmax=1.0, movlim=0.2):
        a, b = np.zeros(self.ne), np.zeros(self.ne)
        lib().or_mma_set_outer_movelimit(self.h, Xmin, Xmax, movlim, np.ascontiguousarray(x, dtype=np.float64),
                                         a, b)
        return a, b

    def mma_update(self, x, dfdx, gx, dgdx, xmin, xmax):
        xv = np.ascontiguousarray(x, dtype=np.float64).copy()
        f = lambda a: np.ascontiguousarray(a, dtype=np.float64).ravel()
        lib().or_mma_update(self.h, xv, f(dfdx), f(gx), f(dgdx), f(xmin), f(xmax))
        return xv

    def mma_design_change(self, x, xold):
        xo = np.ascontiguousarray(xold, dtype=np.float64).copy()
        ch = lib().or_mma_design_change(self.h, np.ascontiguousarray(x, dtype=np.float64), xo)
        return ch, xo

    def mma_state(self):
        a = [np.zeros(self.ne) for _ in range(4)]
        k = C.c_int()
        lib().or_mma_state(self.h, *[x.ctypes.data for x in a], C.byref(k))
        return a + [k.value]

    def mma_options(self, asyminit=0.5, asymdec=0.7, asyminc=1.2, robust=0, constraint_mod=0):
        lib().or_mma_options(self.h, asyminit, asymdec, asyminc, robust, constraint_mod)

    def mma_restart_set(self, xo1, xo2, U, L, k):
        f = lambda a: np.ascontiguousarray(a, dtype=np.float64).ravel()
        lib().or_mma_restart_set(self.h, f(xo1), f(xo2), f(U), f(L), k)

    def mma_kkt(self, x, dfdx, gx, dgdx, xmin, xmax):
        f = lambda a: np.ascontiguousarray(a, dtype=np.float64).ravel()
        n2, ni = C.c_double(), C.c_double()
        lib().or_mma_kkt_residual(self.h, f(x), f(dfdx), f(gx), f(dgdx), f(xmin), f(xmax), C.byref(n2),
                                  C.byref(ni))
        return n2.value, ni.value

    def amg_aggregates(self, level):
        nnode = self.nn if level == 0 else None
        buf = np.zeros(max(self.nn, 1), dtype=np.int32)
        na = lib().or_amg_aggregates(self.h, level, buf)
        return na, buf

    def run(self, maxItr, ch_tol=0.01):
        hist = np.zeros(3 * maxItr)
        xp = np.zeros(self.ne)
        it = lib().or_run(self.h, maxItr, ch_tol, hist, xp)
        return hist.reshape(-1, 3)[:it], xp
