// abi.cu -- the extern "C" boundary (include/topo.h) and the main.cpp loop.
// Every entry point validates its arguments, runs on the context's stream and
// returns a status code; no C++ exception crosses the boundary.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <new>
#include <sstream>
#include <string>
#include <vector>

#include "ctx.h"

namespace topo {
const char* last_error();
int kmatvec64r(Ctx& c, const double* u, double* y, const double* b);

// ----------------------------------------------------------------- small kernels
__global__ void k_fill(long n, double* __restrict__ x, double v) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) x[i] = v;
}
__global__ void k_filter_diag(int nn, int nen, int nkf, const int* __restrict__ n2e_ptr, const int* __restrict__ n2e,
                              const double* __restrict__ kf, double* __restrict__ dinv) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    double s = 0.0;
    for (int p = n2e_ptr[i]; p < n2e_ptr[i + 1]; p++) {
        int q = n2e[p], e = q / nen, l = q % nen;
        int k = l * nen - (l * (l - 1)) / 2;  // packed (l, l)
        s += kf[((size_t)(e >> 5) * nkf + k) * 32 + (e & 31)];
    }
    dinv[i] = s != 0.0 ? 1.0 / s : 1.0;
}
// HeavisideFilter (PDEFilter.cpp:271-279); beta from the argument, or from
// device memory (beta_dev) in the device-driven step
__global__ void k_heaviside(int n, const double* __restrict__ xf, double* __restrict__ xp, double beta, double x0,
                            double Xmin, const double* __restrict__ beta_dev) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (beta_dev) beta = *beta_dev;
    double v = (tanh(beta * x0) + tanh(beta * (xf[i] - x0))) / (tanh(beta * x0) + tanh(beta * (1 - x0)));
    if (v < Xmin) v = Xmin;
    xp[i] = v;
}
// ComputeProjectedSens (PDEFilter.cpp:309-333)
__global__ void k_projsens(int n, int m, const double* __restrict__ xf, double* __restrict__ df, double* __restrict__ dg,
                           double beta, double x0, const double* __restrict__ beta_dev) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (beta_dev) beta = *beta_dev;
    double t = tanh(beta * (xf[i] - x0));
    double dx = beta * (1.0 - pow(t, 2.0)) / (tanh(beta * x0) + tanh(beta * (1 - x0)));
    df[i] = df[i] * dx;
    for (int j = 0; j < m; j++) dg[(long)j * n + i] = dg[(long)j * n + i] * dx;
}

// HeavisideFilter's beta schedule (PDEFilter.cpp:260-268) on the device
__global__ void k_beta_schedule(const int* __restrict__ itr, double beta0, double betamax, double* __restrict__ beta,
                                double* __restrict__ beta_tmp) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int it = *itr;
    if (it < 30) *beta = beta0;
    else if (it % 10 == 0) *beta = fmin(betamax, *beta_tmp + 1);
    *beta_tmp = *beta;
}

// ----------------------------------------------------------------- internal stages
static int sum_device(Ctx& c, const double* v, long n, double* host_out) {
    TRET(finalize_sum(c, v, (int)n, 1, c.dsc.p + DS_TMP));
    TCK(cudaMemcpyAsync(c.hsc.h + 250, c.dsc.p + DS_TMP, sizeof(double), cudaMemcpyDeviceToHost, c.s));
    TCK(cudaStreamSynchronize(c.s));
    *host_out = c.hsc.h[250];
    return 0;
}

int filter_apply(Ctx& c, const double* x, double* xf, double Xmin) {
    TRET(filter_tf(c, x, c.TX.p));
    int its = 0;
    int rc = filter_cg(c, c.TX.p, c.RX.p, &its, 0);
    c.info.filter_its[0] = its;
    TRET(rc);
    TRET(filter_tfxT(c, c.RX.p, xf, true, Xmin));
    return rc;
}

int filter_sens(Ctx& c, double* df, double* dg, int m) {
    int rc = 0, its = 0;
    TRET(filter_tf(c, df, c.TX.p));
    int r = filter_cg(c, c.TX.p, c.RX.p, &its, 1);
    TRET(r);
    rc = std::max(rc, r);
    c.info.filter_its[1] = its;
    TRET(filter_tfxT(c, c.RX.p, df, false, 0.0));
    for (int j = 0; j < m; j++) {
        double* dj = dg + (size_t)j * c.ne;
        TRET(filter_tf(c, dj, c.TX.p));
        r = filter_cg(c, c.TX.p, c.RX.p, &its, std::min(j + 2, 3));
        TRET(r);
        rc = std::max(rc, r);
        if (j + 2 < 4) c.info.filter_its[j + 2] = its;
        TRET(filter_tfxT(c, c.RX.p, dj, false, 0.0));
    }
    return rc;
}

int heaviside(Ctx& c, const double* xf, double* xp, double x0, double beta0, double betamax, int itr, double Xmin,
              int proj) {
    if (!proj) {  // VecCopy(XFiled, XPhys)
        TCK(cudaMemcpyAsync(xp, xf, sizeof(double) * c.ne, cudaMemcpyDeviceToDevice, c.s));
        return 0;
    }
    if (c.sg.dd) {
        // the same beta schedule on the device, from the device's itr
        k_beta_schedule<<<1, 32, 0, c.s>>>(c.di.p + DI_ITR, beta0, betamax, c.dsc.p + DS_BETA, c.dsc.p + DS_BETA_TMP),
            note_launch();
        k_heaviside<<<(c.ne + 255) / 256, 256, 0, c.s>>>(c.ne, xf, xp, 0.0, x0, Xmin, c.dsc.p + DS_BETA), note_launch();
        TCK(cudaGetLastError());
        return 0;
    }
    if (itr < 30) c.beta_proj = beta0;
    else if (itr % 10 == 0) c.beta_proj = std::min(betamax, c.beta_tmp + 1);
    k_heaviside<<<(c.ne + 255) / 256, 256, 0, c.s>>>(c.ne, xf, xp, c.beta_proj, x0, Xmin, nullptr), note_launch();
    c.beta_tmp = c.beta_proj;
    TCK(cudaGetLastError());
    return 0;
}

int projected_sens(Ctx& c, const double* xf, double* df, double* dg, int m, double x0) {
    k_projsens<<<(c.ne + 255) / 256, 256, 0, c.s>>>(c.ne, m, xf, df, dg, c.beta_proj, x0,
                                                    c.sg.dd ? c.dsc.p + DS_BETA : nullptr), note_launch();
    TCK(cudaGetLastError());
    return 0;
}

// ComputeObjectiveAndSensitivities with fx, gx left on the device (dsc)
int fem_obj_sens_dev(Ctx& c, const double* xphys, double* dfdx, double* dgdx) {
    if (!c.U.p) TRET(c.U.alloc((size_t)c.ncases * c.ndof));
    int rc = fem_solve(c, xphys, c.U.p);
    TRET(rc);
    TRET(fem_sensitivities(c, xphys, dfdx, dgdx));
    return rc;
}

static int opt_alloc(Ctx& c) {
    if (c.X.p) return 0;
    const int n = c.ne;
    TRET(c.X.alloc(n)); TRET(c.Xold.alloc(n)); TRET(c.XF.alloc(n)); TRET(c.XP.alloc(n));
    TRET(c.dfdx.alloc(n)); TRET(c.dgdx.alloc((size_t)n * c.p.m)); TRET(c.xmin.alloc(n)); TRET(c.xmax.alloc(n));
    return 0;
}

static float ev_ms(cudaEvent_t a, cudaEvent_t b) {
    float t = 0.f;
    if (cudaEventElapsedTime(&t, a, b) != cudaSuccess) { cudaGetLastError(); t = 0.f; }
    return t;
}

// one pass of main.cpp:72-112
int opt_step(Ctx& c) {
    const topo_params& p = c.p;
    if (p.step_graph) {
        bool ok = false;
        TRET(opt_step_graph_prepare(c, &ok));
        if (ok) {
            for (int part = 0; part < 3; part++) TRET(opt_step_graph_part(c, part));
            return opt_step_graph_finish(c);
        }
    } else {
        c.info.step_graph = 0;
    }
    c.sg.state_dirty = true;  // the host-side itr and beta move on
    c.itr++;
    cudaEventRecord(c.ev[0], c.s);
    int rc_fem = fem_obj_sens_dev(c, c.XP.p, c.dfdx.p, c.dgdx.p);
    TRET(rc_fem);
    cudaEventRecord(c.ev[1], c.s);
    if (p.proj) TRET(projected_sens(c, c.XF.p, c.dfdx.p, c.dgdx.p, p.m, p.x0));
    int rc_f = filter_sens(c, c.dfdx.p, c.dgdx.p, p.m);
    TRET(rc_f);
    cudaEventRecord(c.ev[2], c.s);
    TRET(mma_movelimit(c, p.Xmin, p.Xmax, p.movlim, c.X.p, c.xmin.p, c.xmax.p));
    TRET(mma_update(c, c.X.p, c.dfdx.p, c.dsc.p + DS_GX, c.dgdx.p, c.xmin.p, c.xmax.p));
    TRET(mma_design_change(c, c.X.p, c.Xold.p, c.dsc.p + DS_CH));
    cudaEventRecord(c.ev[3], c.s);
    int rc_f2 = filter_apply(c, c.X.p, c.XF.p, p.Xmin);
    TRET(rc_f2);
    TRET(heaviside(c, c.XF.p, c.XP.p, p.x0, p.beta0, p.betamax, c.itr, p.Xmin, p.proj));
    TCK(cudaMemcpyAsync(c.hsc.h + 240, c.dsc.p, 9 * sizeof(double), cudaMemcpyDeviceToHost, c.s));
    TCK(cudaStreamSynchronize(c.s));
    c.info.last_fx = c.hsc.h[240 + DS_FX];
    c.info.last_gx0 = c.hsc.h[240 + DS_GX];
    c.ch = c.info.last_ch = c.hsc.h[240 + DS_CH];
    c.info.t_fem_ms = ev_ms(c.ev[0], c.ev[1]);
    c.info.t_filter_ms = ev_ms(c.ev[1], c.ev[2]);
    c.info.t_mma_ms = ev_ms(c.ev[2], c.ev[3]);
    if (p.verbose)
        printf("It.: %i, fx: %f, gx[0]: %f, ch.: %f, time: %f\n", c.itr, c.info.last_fx, c.info.last_gx0, c.ch,
               (c.info.t_fem_ms + c.info.t_filter_ms + c.info.t_mma_ms) * 1e-3);
    if (!std::isfinite(c.info.last_fx)) { set_error("compliance is not finite"); return TOPO_ERR_NAN; }
    return std::max(std::max(rc_fem, rc_f), rc_f2);
}

int opt_init(Ctx& c) {
    TRET(opt_alloc(c));
    TRET(mma_alloc(c));
    const int n = c.ne;
    for (double* v : {c.X.p, c.XF.p, c.XP.p, c.Xold.p}) k_fill<<<grid_for(n, 256), 256, 0, c.s>>>(n, v, c.p.volfrac), note_launch();
    TCK(cudaGetLastError());
    c.itr = 0;
    c.ch = 1.0;
    // a fresh optimisation: MMA history, filter warm start and beta state
    // start over as in a new process (MMA.cpp:178-224, PDEFilter.cpp:64-67)
    TCK(cudaMemsetAsync(c.di.p + DI_MMA_K, 0, sizeof(int), c.s));
    c.u_valid = false;
    for (DBuf<double>* b : {&c.xo1, &c.xo2, &c.L, &c.Uas, &c.RX}) TRET(b->zero(c.s));
    c.beta_proj = c.beta_tmp = c.p.beta0;
    TRET(amg_reset_warm_start(c));
    TRET(filter_apply(c, c.X.p, c.XF.p, c.p.Xmin));
    TRET(heaviside(c, c.XF.p, c.XP.p, c.p.x0, c.p.beta0, c.p.betamax, c.itr, c.p.Xmin, c.p.proj));
    c.opt_ready = true;
    return 0;
}

int create(Ctx& c, int nen, int n_nodes, const double* vertex, int n_elems, const int32_t* element, int n_fixed,
           const int32_t* fixed, int n_cases, const int32_t* case_ptr, const int32_t* load_dofs,
           const double* load_vals) {
    c.nen = nen;
    c.nn = n_nodes;
    c.ne = n_elems;
    for (int i = 0; i < 4; i++) TCK(cudaEventCreate(&c.ev[i]));
    TRET(c.dsc.alloc(DS_COUNT));
    TRET(c.dsc.zero(c.s));
    TRET(c.di.alloc(DI_COUNT));
    TRET(c.di.zero(c.s));
    TRET(c.hsc.alloc(1024));
    TRET(build_mesh(c, vertex, element, n_fixed, fixed, n_cases, case_ptr, load_dofs, load_vals));
    TRET(elem_setup(c));
    TRET(sum_device(c, c.vol.p, c.ne, &c.TV));
    // filter: Jacobi diagonal of KF, work vectors, RX = 0 (VecDuplicate)
    TRET(c.fdiag_inv.alloc(c.nn));
    k_filter_diag<<<(c.nn + 255) / 256, 256, 0, c.s>>>(c.nn, c.nen, c.nkf, c.n2e_ptr.p, c.n2e.p, c.kf.p, c.fdiag_inv.p), note_launch();
    TCK(cudaGetLastError());
    for (DBuf<double>* b : {&c.RX, &c.TX, &c.fr, &c.fz, &c.fp, &c.fw}) { TRET(b->alloc(c.nn)); TRET(b->zero(c.s)); }
    TRET(build_amg_host(c));
    TRET(amg_alloc(c));
    if (c.p.deterministic) TRET(c.det_scr.alloc((size_t)c.ntiles * 32 * c.nde));  // per-element contributions
    // completion counter of the reductions that finish in their last block
    // (allocated here, never inside a graph capture)
    TRET(c.red_count.alloc(1));
    TCK(cudaMemsetAsync(c.red_count.p, 0, sizeof(unsigned), c.s));
    TRET(mma_alloc(c));
    TCK(cudaStreamSynchronize(c.s));
    return 0;
}

// ----------------------------------------------------------------- generator (host)
static uint64_t sm64(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
static double sm64_unit(uint64_t& s) { return (double)(sm64(s) >> 11) * (1.0 / 9007199254740992.0); }

}  // namespace topo

using namespace topo;

#define GUARD_BEGIN try {
#define GUARD_END                                                  \
    }                                                              \
    catch (const std::bad_alloc&) {                                \
        set_error("host allocation failed");                       \
        return TOPO_ERR_OOM;                                       \
    }                                                              \
    catch (...) {                                                  \
        set_error("unexpected internal exception");                \
        return TOPO_ERR_CUDA;                                      \
    }

struct topo_ctx {
    Ctx c;
};

namespace topo {
cudaEvent_t prof_event(Ctx& c) {
    if (c.prof.pool.empty()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) { cudaGetLastError(); return nullptr; }
        return e;
    }
    cudaEvent_t e = c.prof.pool.back();
    c.prof.pool.pop_back();
    return e;
}
}  // namespace topo

extern "C" {

const char* topo_last_error(void) { return topo::last_error(); }
const char* topo_version(void) { return "topo-b200 1.0 (sm_100a)"; }

int topo_struct_sizes(size_t* params_bytes, size_t* info_bytes) {
    if (params_bytes) *params_bytes = sizeof(topo_params);
    if (info_bytes) *info_bytes = sizeof(topo_solve_info);
    return 0;
}

void topo_params_default(topo_params* p) {
    if (!p) return;
    memset(p, 0, sizeof(*p));
    p->Emin = 1.0e-9; p->Emax = 1.0e6; p->nu = 0.3; p->penal = 3.0; p->volfrac = 0.12; p->rmin = 0.01;
    p->Xmin = 0.01; p->Xmax = 1.0; p->movlim = 0.2; p->x0 = 0.5; p->beta0 = 1.0; p->betamax = 8.0;
    p->proj = 0; p->maxItr = 200; p->m = 1; p->ch_tol = 0.01;
    p->fem_rtol = 1.0e-5; p->fem_restart = 30; p->fem_maxit = 10000;
    p->precision = TOPO_PREC_FP64; p->amg_max_levels = 8; p->amg_coarse_max = 100; p->amg_smooth_p = 1;
    p->cheb_degree = 2; p->fine_smoother_matfree = 0;
    p->filter_rtol = 1.0e-5; p->filter_atol = 1.0e-50; p->filter_dtol = 1.0e5; p->filter_maxit = 10000;
    p->verbose = 0;
    p->amg_rho_its = 10;
    p->cheb_safety = 1.0;
    p->fem_warm_start = 0;
    p->fem_block = 1;
    p->fem_graphs = 1;
    p->cheb_degree_post = 0;
    p->cheb_degree_coarse = 4;
    p->amg_half_fine = 0;
    p->amg_coarse_cta = 0;
    p->autotune = 1;
    p->pdl = 1;
    p->step_graph = 0;
    p->deterministic = 0;
}

int topo_device_alloc(size_t bytes, void** ptr) {
    if (!ptr) { set_error("null output pointer"); return TOPO_ERR_ARG; }
    cudaError_t e = cudaMalloc(ptr, bytes ? bytes : 1);
    if (e != cudaSuccess) { cudaGetLastError(); *ptr = nullptr; return cuda_fail(e, __FILE__, __LINE__); }
    return 0;
}
int topo_device_free(void* ptr) {
    if (ptr) TCK(cudaFree(ptr));
    return 0;
}
int topo_memcpy_h2d(void* dst, const void* src, size_t bytes, topo_ctx* ctx) {
    if (!dst || !src) { set_error("null pointer"); return TOPO_ERR_ARG; }
    cudaStream_t s = ctx ? ctx->c.s : nullptr;
    TCK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
    TCK(cudaStreamSynchronize(s));
    return 0;
}
int topo_memcpy_d2h(void* dst, const void* src, size_t bytes, topo_ctx* ctx) {
    if (!dst || !src) { set_error("null pointer"); return TOPO_ERR_ARG; }
    cudaStream_t s = ctx ? ctx->c.s : nullptr;
    TCK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
    TCK(cudaStreamSynchronize(s));
    return 0;
}
int topo_sync(topo_ctx* ctx) {
    if (!ctx) { set_error("null context"); return TOPO_ERR_ARG; }
    TCK(cudaStreamSynchronize(ctx->c.s));
    return 0;
}

static int check_params(const topo_params* p) {
    if (!(p->Emax > 0) || !(p->Emin >= 0) || !(p->penal > 0) || !(p->rmin > 0) || !(p->nu > -1 && p->nu < 0.5)) {
        set_error("invalid material/filter parameters");
        return TOPO_ERR_ARG;
    }
    if (p->m < 1 || p->m > kMaxM) { set_error("m must be in [1,%d]", kMaxM); return TOPO_ERR_ARG; }
    if (p->fem_restart < 1 || p->fem_restart > 128) { set_error("fem_restart must be in [1,128]"); return TOPO_ERR_ARG; }
    if (p->cheb_degree < 1 || p->cheb_degree > 15) { set_error("cheb_degree must be in [1,15]"); return TOPO_ERR_ARG; }
    if (p->precision != TOPO_PREC_FP64 && p->precision != TOPO_PREC_MIXED) { set_error("bad precision"); return TOPO_ERR_ARG; }
    if (p->amg_coarse_max < 6 || p->amg_coarse_max > 4000) { set_error("amg_coarse_max must be in [6,4000]"); return TOPO_ERR_ARG; }
    if (p->amg_max_levels < 1 || p->amg_max_levels > kMaxLevels) {
        set_error("amg_max_levels must be in [1,%d]", kMaxLevels);
        return TOPO_ERR_ARG;
    }
    if (p->cheb_degree_post < 0 || p->cheb_degree_post > 15 || p->cheb_degree_coarse < 0 || p->cheb_degree_coarse > 15) {
        set_error("cheb_degree_post and cheb_degree_coarse must be in [0,15] (0: as cheb_degree)");
        return TOPO_ERR_ARG;
    }
    if (p->blk_stages != 0 && p->blk_stages != 2 && p->blk_stages != 3) {
        set_error("blk_stages must be 0 (tuned), 2 or 3");
        return TOPO_ERR_ARG;
    }
    if (p->amg_rho_its < 0 || p->amg_rho_its > 1000) { set_error("amg_rho_its must be in [0,1000]"); return TOPO_ERR_ARG; }
    if (!(p->cheb_safety >= 0.0 && p->cheb_safety <= 10.0)) {
        set_error("cheb_safety must be in [0,10] (0: 1)");
        return TOPO_ERR_ARG;
    }
    const struct { int v; const char* name; } flags[] = {
        {p->proj, "proj"}, {p->amg_smooth_p, "amg_smooth_p"}, {p->fine_smoother_matfree, "fine_smoother_matfree"},
        {p->fem_warm_start, "fem_warm_start"}, {p->fem_block, "fem_block"}, {p->fem_graphs, "fem_graphs"},
        {p->autotune, "autotune"}, {p->amg_coarse_cta, "amg_coarse_cta"}, {p->amg_half_fine, "amg_half_fine"},
        {p->pdl, "pdl"}, {p->step_graph, "step_graph"}, {p->deterministic, "deterministic"}};
    for (const auto& f : flags)
        if (f.v != 0 && f.v != 1) { set_error("%s must be 0 or 1", f.name); return TOPO_ERR_ARG; }
    return 0;
}

int topo_create(const topo_params* p, int nen, int n_nodes, const double* vertex, int n_elems, const int32_t* element,
                int n_fixed, const int32_t* fixed_dofs, int n_cases, const int32_t* case_ptr, const int32_t* load_dofs,
                const double* load_vals, void* stream, topo_ctx** out) {
    GUARD_BEGIN
    if (!out) { set_error("null output pointer"); return TOPO_ERR_ARG; }
    *out = nullptr;
    if (nen != 8 && nen != 4) { set_error("nen must be 8 (hex8) or 4 (tet4)"); return TOPO_ERR_ARG; }
    if (n_nodes <= 0 || n_elems <= 0 || !vertex || !element) { set_error("empty mesh"); return TOPO_ERR_MESH; }
    if (n_fixed < 0 || (n_fixed > 0 && !fixed_dofs)) { set_error("bad fixed DOF list"); return TOPO_ERR_ARG; }
    if (n_cases < 1 || n_cases > kMaxCases || !case_ptr) { set_error("n_cases must be in [1,%d]", kMaxCases); return TOPO_ERR_ARG; }
    if (case_ptr[n_cases] > 0 && (!load_dofs || !load_vals)) { set_error("null load arrays"); return TOPO_ERR_ARG; }
    if ((long)n_nodes * 3 >= (1L << 31) || (long)n_elems * nen >= (1L << 31)) { set_error("mesh too large for 32-bit ids"); return TOPO_ERR_ARG; }
    topo_params pp;
    if (p) pp = *p;
    else topo_params_default(&pp);
    TRET(check_params(&pp));
    // host-side validation first, so a corrupt mesh is reported as such
    // whether or not a device is present
    for (long q = 0; q < 3L * n_nodes; q++)
        if (!std::isfinite(vertex[q])) { set_error("vertex %ld is not finite", q / 3); return TOPO_ERR_MESH; }
    for (long q = 0; q < (long)n_elems * nen; q++)
        if (element[q] < 0 || element[q] >= n_nodes) {
            set_error("element %ld references node %d outside [0,%d)", q / nen, element[q], n_nodes);
            return TOPO_ERR_MESH;
        }
    for (int i = 0; i < n_fixed; i++)
        if (fixed_dofs[i] < 0 || fixed_dofs[i] >= 3 * n_nodes) { set_error("fixed DOF %d out of range", fixed_dofs[i]); return TOPO_ERR_MESH; }
    if (case_ptr[0] != 0) { set_error("case_ptr[0] must be 0"); return TOPO_ERR_ARG; }
    for (int k = 0; k < n_cases; k++) {
        if (case_ptr[k + 1] < case_ptr[k]) { set_error("case_ptr not monotone"); return TOPO_ERR_ARG; }
        for (int q = case_ptr[k]; q < case_ptr[k + 1]; q++)
            if (load_dofs[q] < 0 || load_dofs[q] >= 3 * n_nodes || !std::isfinite(load_vals[q])) {
                set_error("load entry %d invalid (DOF %d)", q, load_dofs[q]);
                return TOPO_ERR_MESH;
            }
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        set_error("no CUDA device: this library has no CPU fallback");
        return TOPO_ERR_CUDA;
    }
    topo_ctx* t = new topo_ctx();
    t->c.p = pp;
    if (stream) t->c.s = (cudaStream_t)stream;
    else {
        cudaError_t e = cudaStreamCreateWithFlags(&t->c.s, cudaStreamNonBlocking);
        if (e != cudaSuccess) { delete t; return cuda_fail(e, __FILE__, __LINE__); }
        t->c.own_stream = true;
    }
    int rc = create(t->c, nen, n_nodes, vertex, n_elems, element, n_fixed, fixed_dofs, n_cases, case_ptr, load_dofs,
                    load_vals);
    if (rc < 0) {
        std::string msg = topo::last_error();
        topo_destroy(t);
        set_error("%s", msg.c_str());
        return rc;
    }
    *out = t;
    return 0;
    GUARD_END
}

int topo_destroy(topo_ctx* ctx) {
    if (!ctx) return 0;
    cudaStreamSynchronize(ctx->c.s);
    step_batch_forget(&ctx->c);
    cudaGetLastError();
    for (int i = 0; i < 4; i++)
        if (ctx->c.ev[i]) cudaEventDestroy(ctx->c.ev[i]);
    for (auto e : ctx->c.prof.pool) cudaEventDestroy(e);
    for (auto e : ctx->c.gm_ev) cudaEventDestroy(e);
    for (auto& r : ctx->c.prof.rec)
        for (auto& pr : r) { cudaEventDestroy(pr.first); cudaEventDestroy(pr.second); }
    cudaStream_t s = ctx->c.s;
    bool own = ctx->c.own_stream;
    delete ctx;
    if (own) cudaStreamDestroy(s);
    return 0;
}

int topo_get_params(topo_ctx* ctx, topo_params* p) {
    if (!ctx || !p) { set_error("null argument"); return TOPO_ERR_ARG; }
    *p = ctx->c.p;
    return 0;
}
int topo_set_params(topo_ctx* ctx, const topo_params* p) {
    if (!ctx || !p) { set_error("null argument"); return TOPO_ERR_ARG; }
    TRET(check_params(p));
    const topo_params& o = ctx->c.p;
    if (p->nu != o.nu || p->rmin != o.rmin || p->m != o.m || p->amg_max_levels != o.amg_max_levels ||
        p->amg_coarse_max != o.amg_coarse_max || p->amg_smooth_p != o.amg_smooth_p || p->fem_restart != o.fem_restart ||
        p->deterministic != o.deterministic) {
        set_error("nu, rmin, m, restart, AMG structure options and deterministic are fixed at creation");
        return TOPO_ERR_ARG;
    }
    ctx->c.p = *p;
    return 0;
}
int topo_sizes(topo_ctx* ctx, int* nen, int* n_nodes, int* n_elems, int* n_cases) {
    if (!ctx) { set_error("null context"); return TOPO_ERR_ARG; }
    if (nen) *nen = ctx->c.nen;
    if (n_nodes) *n_nodes = ctx->c.nn;
    if (n_elems) *n_elems = ctx->c.ne;
    if (n_cases) *n_cases = ctx->c.ncases;
    return 0;
}
void* topo_stream(topo_ctx* ctx) { return ctx ? (void*)ctx->c.s : nullptr; }

// ---------------------------------------------------------------- SolveFem
int topo_fem_volumes(topo_ctx* ctx, double* vol_d, double* tv) {
    if (!ctx) { set_error("null context"); return TOPO_ERR_ARG; }
    Ctx& c = ctx->c;
    if (vol_d) TCK(cudaMemcpyAsync(vol_d, c.vol.p, sizeof(double) * c.ne, cudaMemcpyDeviceToDevice, c.s));
    if (tv) *tv = c.TV;
    TCK(cudaStreamSynchronize(c.s));
    return 0;
}

int topo_fem_element_matrix(topo_ctx* ctx, int e, double* ke) {
    if (!ctx || !ke) { set_error("null argument"); return TOPO_ERR_ARG; }
    Ctx& c = ctx->c;
    if (e < 0 || e >= c.ne) { set_error("element index out of range"); return TOPO_ERR_ARG; }
    GUARD_BEGIN
    const int nd = c.nde, npk = c.npk;
    std::vector<double> pk(npk);
    const size_t base = (size_t)(e >> 5) * npk * 32 + (e & 31);
    TCK(cudaMemcpy2DAsync(pk.data(), sizeof(double), c.ke64.p + base, 32 * sizeof(double), sizeof(double), npk,
                          cudaMemcpyDeviceToHost, c.s));
    TCK(cudaStreamSynchronize(c.s));
    int k = 0;
    for (int i = 0; i < nd; i++)
        for (int j = i; j < nd; j++, k++) { ke[i * nd + j] = pk[k]; ke[j * nd + i] = pk[k]; }
    return 0;
    GUARD_END
}

int topo_fem_apply(topo_ctx* ctx, const double* xphys_d, const double* u_d, double* y_d) {
    if (!ctx || !xphys_d || !u_d || !y_d) { set_error("null argument"); return TOPO_ERR_ARG; }
    GUARD_BEGIN
    Ctx& c = ctx->c;
    TRET(compute_moduli(c, xphys_d));
    TRET(kmatvec(c, c.Ee64.p, u_d, y_d));
    TCK(cudaStreamSynchronize(c.s));
    return 0;
    GUARD_END
}

int topo_fem_apply_block(topo_ctx* ctx, const double* xphys_d, const double* u_d, double* y_d) {
    if (!ctx || !xphys_d || !u_d || !y_d) { set_error("null argument"); return TOPO_ERR_ARG; }
    GUARD_BEGIN
    Ctx& c = ctx->c;
    TRET(compute_moduli(c, xphys_d));
    TRET(blk_setup(c));
    const size_t nf = (size_t)c.ndof * c.blk.kb;
    DBuf<double> ub, yb;
    TRET(ub.alloc(nf));
    TRET(yb.alloc(nf));
    TRET(blk_interleave(c, u_d, ub.p));
    TRET(blk_apply(c, ub.p, yb.p, nullptr, 1.0));
    TRET(blk_deinterleave(c, yb.p, y_d));
    TCK(cudaStreamSynchronize(c.s));
    TRET(blk_check_error(c));
    return 0;
    GUARD_END
}

int topo_fem_obj_sens(topo_ctx* ctx, const double* xphys_d, double* fx, double* gx, double* dfdx_d, double* dgdx_d) {
    if (!ctx || !xphys_d || !fx || !gx || !dfdx_d || !dgdx_d) { set_error("null argument"); return TOPO_ERR_ARG; }
    GUARD_BEGIN
    Ctx& c = ctx->c;
    int rc = fem_obj_sens_dev(c, xphys_d, dfdx_d, dgdx_d);
    TRET(rc);
    TCK(cudaMemcpyAsync(c.hsc.h + 240, c.dsc.p, (DS_GX + c.p.m) * sizeof(double), cudaMemcpyDeviceToHost, c.s));
    TCK(cudaStreamSynchronize(c.s));
    *fx = c.hsc.h[240 + DS_FX];
    for (int j = 0; j < c.p.m; j++) gx[j] = c.hsc.h[240 + DS_GX + j];
    return rc;
    GUARD_END
}

int topo_fem_solve(topo_ctx* ctx, const double* xphys_d, double* u_d) {
    if (!ctx || !xphys_d) { set_error("null argument"); return TOPO_ERR_ARG; }
    GUARD_BEGIN
    Ctx& c = ctx->c;
    if (!c.U.p) TRET(c.U.alloc((size_t)c.ncases * c.ndof));
    int rc = fem_solve(c, xphys_d, c.U.p);
    TRET(rc);
    if (u_d) TCK(cudaMemcpyAsync(u_d, c.U.p, sizeof(double) * c.ncases * c.ndof, cudaMemcpyDeviceToDevice, c.s));
    TCK(cudaStreamSynchronize(c.s));
    return rc;
    GUARD_END
}

int topo_fem_displacement(topo_ctx* ctx, double* u_d) {
    if (!ctx || !u_d) { set_error("null argument"); return TOPO_ERR_ARG; }
    Ctx& c = ctx->c;
    if (!c.U.p) { set_error("no displacement computed yet"); return TOPO_ERR_ARG; }
    TCK(cudaMemcpyAsync(u_d, c.U.p, sizeof(double) * c.ncases * c.ndof, cudaMemcpyDeviceToDevice, c.s));
    TCK(cudaStreamSynchronize(c.s));
    return 0;
}

int topo_fem_von_mises(topo_ctx* ctx, const double* xphys_d, double* vms_d) {
    if (!ctx || !xphys_d || !vms_d) { set_error("null argument"); return TOPO_ERR_ARG; }
    Ctx& c = ctx->c;
    if (!c.U.p) { set_error("no displacement computed yet"); return TOPO_ERR_ARG; }
    TRET(von_mises(c, xphys_d, vms_d));
    TCK(cudaStreamSynchronize(c.s));
    return 0;
}

// ---------------------------------------------------------------- PDEFilter
int topo_filter_apply(topo_ctx* ctx, const double* x_d, double* xf_d, double Xmin) {
    if (!ctx || !x_d || !xf_d) { set_error("null argument"); return TOPO_ERR_ARG; }
    GUARD_BEGIN
    int rc = filter_apply(ctx->c, x_d, xf_d, Xmin);
    TRET(rc);
    TCK(cudaStreamSynchronize(ctx->c.s));
    return rc;
    GUARD_END
}
int topo_filter_sens(topo_ctx* ctx, double* dfdx_d, double* dgdx_d, int m) {
    if (!ctx || !dfdx_d || (m > 0 && !dgdx_d) || m < 0) { set_error("bad argument"); return TOPO_ERR_ARG; }
    GUARD_BEGIN
    int rc = filter_sens(ctx->c, dfdx_d, dgdx_d, m);
    TRET(rc);
    TCK(cudaStreamSynchronize(ctx->c.s));
    return rc;
    GUARD_END
}
int topo_heaviside(topo_ctx* ctx, const double* xf_d, double* xp_d, double x0, double beta0, double betamax, int itr,
                   double Xmin, int proj) {
    if (!ctx || !xf_d || !xp_d) { set_error("null argument"); return TOPO_ERR_ARG; }
    TRET(heaviside(ctx->c, xf_d, xp_d, x0, beta0, betamax, itr, Xmin, proj));
    TCK(cudaStreamSynchronize(ctx->c.s));
    return 0;
}
int topo_projected_sens(topo_ctx* ctx, const double* xf_d, double* dfdx_d, double* dgdx_d, int m, double x0) {
    if (!ctx || !xf_d || !dfdx_d || (m > 0 && !dgdx_d)) { set_error("null argument"); return TOPO_ERR_ARG; }
    TRET(projected_sens(ctx->c, xf_d, dfdx_d, dgdx_d, m, x0));
    TCK(cudaStreamSynchronize(ctx->c.s));
    return 0;
}
int topo_filter_state(topo_ctx* ctx, double* rx_d, int set) {
    if (!ctx || !rx_d) { set_error("null argument"); return TOPO_ERR_ARG; }
    Ctx& c = ctx->c;
    if (set) TCK(cudaMemcpyAsync(c.RX.p, rx_d, sizeof(double) * c.nn, cudaMemcpyDeviceToDevice, c.s));
    else TCK(cudaMemcpyAsync(rx_d, c.RX.p, sizeof(double) * c.nn, cudaMemcpyDeviceToDevice, c.s));
    TCK(cudaStreamSynchronize(c.s));
    return 0;
}

// ---------------------------------------------------------------- MMA
int topo_mma_set_outer_movelimit(topo_ctx* ctx, double Xmin, double Xmax, double movlim, const double* x_d,
                                 double* xmin_d, double* xmax_d) {
    if (!ctx || !x_d || !xmin_d || !xmax_d) { set_error("null argument"); return TOPO_ERR_ARG; }
    TRET(mma_movelimit(ctx->c, Xmin, Xmax, movlim, x_d, xmin_d, xmax_d));
    TCK(cudaStreamSynchronize(ctx->c.s));
    return 0;
}
int topo_mma_update(topo_ctx* ctx, double* xval_d, const double* dfdx_d, const double* gx, const double* dgdx_d,
                    const double* xmin_d, const double* xmax_d) {
    if (!ctx || !xval_d || !dfdx_d || !gx || !dgdx_d || !xmin_d || !xmax_d) { set_error("null argument"); return TOPO_ERR_ARG; }
    GUARD_BEGIN
    Ctx& c = ctx->c;
    for (int j = 0; j < c.p.m; j++) c.hsc.h[300 + j] = gx[j];
    TCK(cudaMemcpyAsync(c.dsc.p + DS_TMP + 1, c.hsc.h + 300, sizeof(double) * c.p.m, cudaMemcpyHostToDevice, c.s));
    TRET(mma_update(c, xval_d, dfdx_d, c.dsc.p + DS_TMP + 1, dgdx_d, xmin_d, xmax_d));
    TCK(cudaStreamSynchronize(c.s));
    return 0;
    GUARD_END
}
int topo_mma_design_change(topo_ctx* ctx, const double* x_d, double* xold_d, double* ch) {
    if (!ctx || !x_d || !xold_d || !ch) { set_error("null argument"); return TOPO_ERR_ARG; }
    Ctx& c = ctx->c;
    TRET(mma_design_change(c, x_d, xold_d, c.dsc.p + DS_CH));
    TCK(cudaMemcpyAsync(c.hsc.h + 250, c.dsc.p + DS_CH, sizeof(double), cudaMemcpyDeviceToHost, c.s));
    TCK(cudaStreamSynchronize(c.s));
    *ch = c.hsc.h[250];
    return 0;
}
int topo_mma_set_asymptotes(topo_ctx* ctx, double init, double decrease, double increase) {
    if (!ctx) { set_error("null context"); return TOPO_ERR_ARG; }
    ctx->c.asyminit = init;
    ctx->c.asymdec = decrease;
    ctx->c.asyminc = increase;
    return 0;
}
int topo_mma_set_robust_asymptotes_type(topo_ctx* ctx, int val) {
    if (!ctx) { set_error("null context"); return TOPO_ERR_ARG; }
    if (val == 0 || val == 1) ctx->c.robust_type = val;
    else {
        ctx->c.robust_type = 0;
        set_error("RobustAsymptotesType cannot be set to: %d", val);
        return TOPO_ERR_ARG;
    }
    return 0;
}
int topo_mma_constraint_modification(topo_ctx* ctx, int on) {
    if (!ctx) { set_error("null context"); return TOPO_ERR_ARG; }
    ctx->c.constraint_mod = on ? 1 : 0;
    return 0;
}
int topo_mma_restart(topo_ctx* ctx, double* xo1_d, double* xo2_d, double* U_d, double* L_d, int* k, int set) {
    if (!ctx || !xo1_d || !xo2_d || !U_d || !L_d) { set_error("null argument"); return TOPO_ERR_ARG; }
    Ctx& c = ctx->c;
    TRET(mma_alloc(c));
    const size_t b = sizeof(double) * c.ne;
    auto kind = cudaMemcpyDeviceToDevice;
    if (set) {
        TCK(cudaMemcpyAsync(c.xo1.p, xo1_d, b, kind, c.s)); TCK(cudaMemcpyAsync(c.xo2.p, xo2_d, b, kind, c.s));
        TCK(cudaMemcpyAsync(c.Uas.p, U_d, b, kind, c.s)); TCK(cudaMemcpyAsync(c.L.p, L_d, b, kind, c.s));
        if (k) TCK(cudaMemcpyAsync(c.di.p + DI_MMA_K, k, sizeof(int), cudaMemcpyHostToDevice, c.s));
    } else {
        TCK(cudaMemcpyAsync(xo1_d, c.xo1.p, b, kind, c.s)); TCK(cudaMemcpyAsync(xo2_d, c.xo2.p, b, kind, c.s));
        TCK(cudaMemcpyAsync(U_d, c.Uas.p, b, kind, c.s)); TCK(cudaMemcpyAsync(L_d, c.L.p, b, kind, c.s));
        if (k) TCK(cudaMemcpyAsync(k, c.di.p + DI_MMA_K, sizeof(int), cudaMemcpyDeviceToHost, c.s));
    }
    TCK(cudaStreamSynchronize(c.s));
    return 0;
}
int topo_mma_kkt_residual(topo_ctx* ctx, const double* x_d, const double* dfdx_d, const double* gx, const double* dgdx_d,
                          const double* xmin_d, const double* xmax_d, double* norm2, double* norm_inf) {
    if (!ctx || !x_d || !dfdx_d || !gx || !dgdx_d || !xmin_d || !xmax_d || !norm2 || !norm_inf) {
        set_error("null argument");
        return TOPO_ERR_ARG;
    }
    Ctx& c = ctx->c;
    for (int j = 0; j < c.p.m; j++) c.hsc.h[300 + j] = gx[j];
    TCK(cudaMemcpyAsync(c.dsc.p + DS_TMP + 1, c.hsc.h + 300, sizeof(double) * c.p.m, cudaMemcpyHostToDevice, c.s));
    return mma_kkt(c, x_d, dfdx_d, c.dsc.p + DS_TMP + 1, dgdx_d, xmin_d, xmax_d, norm2, norm_inf);
}

int topo_test_block_bank_layout(int nd, int32_t* perm) {
    if (nd != 24 && nd != 12) { set_error("nd must be 24 (hex8) or 12 (tet4)"); return TOPO_ERR_ARG; }
    if (!perm) { set_error("null output pointer"); return TOPO_ERR_ARG; }
    GUARD_BEGIN
    std::vector<int> p;
    const int rc = blk_bank_perm(nd, p);
    for (size_t k = 0; k < p.size(); k++) perm[k] = p[k];
    return rc;
    GUARD_END
}
int topo_test_wait_limits(topo_ctx* ctx, unsigned barrier_spins, unsigned long long copy_cycles, int hold) {
    if (!ctx || (hold != 0 && hold != 1)) { set_error("bad argument"); return TOPO_ERR_ARG; }
    Ctx::WaitLimits d;
    ctx->c.wait.barrier_spins = barrier_spins ? barrier_spins : d.barrier_spins;
    ctx->c.wait.copy_cycles = copy_cycles ? copy_cycles : d.copy_cycles;
    ctx->c.wait.hold = hold;
    return 0;
}

// ---------------------------------------------------------------- main loop
int topo_opt_init(topo_ctx* ctx) {
    if (!ctx) { set_error("null context"); return TOPO_ERR_ARG; }
    GUARD_BEGIN
    TRET(opt_init(ctx->c));
    TCK(cudaStreamSynchronize(ctx->c.s));
    return 0;
    GUARD_END
}
int topo_opt_step(topo_ctx* ctx, int* itr, double* fx, double* gx0, double* ch) {
    if (!ctx) { set_error("null context"); return TOPO_ERR_ARG; }
    GUARD_BEGIN
    Ctx& c = ctx->c;
    if (c.sg.stage) { set_error("a design iteration of this context is still in flight"); return TOPO_ERR_ARG; }
    if (!c.opt_ready) TRET(opt_init(c));
    int rc = opt_step(c);
    TRET(rc);
    if (itr) *itr = c.itr;
    if (fx) *fx = c.info.last_fx;
    if (gx0) *gx0 = c.info.last_gx0;
    if (ch) *ch = c.info.last_ch;
    return rc;
    GUARD_END
}
int topo_opt_run(topo_ctx* ctx, int max_itr, double* hist, int* iterations) {
    if (!ctx) { set_error("null context"); return TOPO_ERR_ARG; }
    GUARD_BEGIN
    Ctx& c = ctx->c;
    if (c.sg.stage) { set_error("a design iteration of this context is still in flight"); return TOPO_ERR_ARG; }
    if (!c.opt_ready) TRET(opt_init(c));
    int worst = 0, done = 0;
    const double tol = c.p.ch_tol;
    while (c.itr < max_itr && (tol <= 0 || c.ch > tol)) {
        int rc = opt_step(c);
        TRET(rc);
        worst = std::max(worst, rc);
        if (hist) {
            hist[3 * done] = c.info.last_fx;
            hist[3 * done + 1] = c.info.last_gx0;
            hist[3 * done + 2] = c.info.last_ch;
        }
        done++;
    }
    if (iterations) *iterations = done;
    return worst;
    GUARD_END
}
int topo_opt_step_batch(topo_ctx* const* ctxs, int n, int* status, double* fx) {
    if (!ctxs || n < 0) { set_error("bad argument"); return TOPO_ERR_ARG; }
    for (int i = 0; i < n; i++)
        if (!ctxs[i]) { set_error("null context %d", i); return TOPO_ERR_ARG; }
    GUARD_BEGIN
    std::vector<int> rc(n, 0);
    std::vector<char> replay(n, 0);
    for (int i = 0; i < n; i++) {
        Ctx& c = ctxs[i]->c;
        if (c.sg.stage) {
            set_error("a design iteration of context %d is still in flight", i);
            rc[i] = TOPO_ERR_ARG;
            continue;
        }
        if (!c.opt_ready) rc[i] = opt_init(c);
        bool ok = false;
        if (rc[i] >= 0 && c.p.step_graph) rc[i] = opt_step_graph_prepare(c, &ok);
        replay[i] = rc[i] >= 0 && ok;
    }
    // the replayed instances' iterations as one graph launch, or, without a
    // batch graph, every instance's own three graphs on its own stream (the
    // cooperative dual solves of part 1 run one after another either way)
    std::vector<Ctx*> rs;
    for (int i = 0; i < n; i++)
        if (replay[i] && rc[i] >= 0) rs.push_back(&ctxs[i]->c);
    bool one = false;
    const int brc = opt_step_graph_batch(rs.data(), (int)rs.size(), &one);
    if (brc < 0) {
        for (int i = 0; i < n; i++)
            if (replay[i] && rc[i] >= 0) rc[i] = brc;
    }
    if (!one)
        for (int part = 0; part < 3; part++)
            for (int i = 0; i < n; i++)
                if (replay[i] && rc[i] >= 0) rc[i] = opt_step_graph_part(ctxs[i]->c, part);
    for (int i = 0; i < n; i++)
        if (!replay[i] && rc[i] >= 0) rc[i] = opt_step(ctxs[i]->c);
    for (int i = 0; i < n; i++)
        if (replay[i] && rc[i] >= 0) rc[i] = opt_step_graph_finish(ctxs[i]->c);
    int worst = 0, err = 0;
    for (int i = 0; i < n; i++) {
        if (status) status[i] = rc[i];
        if (fx) fx[i] = ctxs[i]->c.info.last_fx;
        if (rc[i] < 0 && !err) err = rc[i];
        worst = std::max(worst, rc[i]);
    }
    return err ? err : worst;
    GUARD_END
}

int topo_opt_step_async(topo_ctx* ctx) {
    if (!ctx) { set_error("null context"); return TOPO_ERR_ARG; }
    GUARD_BEGIN
    Ctx& c = ctx->c;
    if (c.sg.stage != 0) { set_error("a design iteration of this context is still in flight"); return TOPO_ERR_ARG; }
    if (!c.opt_ready) TRET(opt_init(c));
    bool ok = false;
    if (c.p.step_graph) TRET(opt_step_graph_prepare(c, &ok));
    if (ok) {
        TRET(opt_step_graph_part(c, 0));
        c.sg.stage = 1;
        return 0;
    }
    const int rc = opt_step(c);  // a direct step: done when this returns
    TRET(rc);
    c.sg.direct_rc = rc;
    c.sg.stage = 3;
    return 0;
    GUARD_END
}

int topo_opt_step_query(topo_ctx* ctx, int* done, int* itr, double* fx, double* gx0, double* ch) {
    if (!ctx || !done) { set_error("null argument"); return TOPO_ERR_ARG; }
    GUARD_BEGIN
    Ctx& c = ctx->c;
    *done = 0;
    int rc = 0;
    switch (c.sg.stage) {
        case 0: set_error("no design iteration of this context was started"); return TOPO_ERR_ARG;
        case 1: {  // the solve part: once it is done, the MMA update and the filter go
            const cudaError_t e = cudaEventQuery(c.sg.p0_done);
            if (e == cudaErrorNotReady) return 0;
            if (e != cudaSuccess) { c.sg.stage = 0; return cuda_fail(e, __FILE__, __LINE__); }
            rc = opt_step_graph_part(c, 1);
            if (rc >= 0) rc = opt_step_graph_part(c, 2);
            if (rc < 0) { c.sg.stage = 0; return rc; }
            c.sg.stage = 2;
            return 0;
        }
        case 2: {
            const cudaError_t e = cudaEventQuery(c.sg.e1);
            if (e == cudaErrorNotReady) return 0;
            c.sg.stage = 0;
            if (e != cudaSuccess) return cuda_fail(e, __FILE__, __LINE__);
            rc = opt_step_graph_finish(c);
            break;
        }
        default:
            c.sg.stage = 0;
            rc = c.sg.direct_rc;
    }
    *done = 1;
    if (itr) *itr = c.itr;
    if (fx) *fx = c.info.last_fx;
    if (gx0) *gx0 = c.info.last_gx0;
    if (ch) *ch = c.info.last_ch;
    return rc;
    GUARD_END
}

int topo_opt_step_host(topo_ctx* ctx, const double* x_in, double* x_out, double* xphys_out, double* fx) {
    if (!ctx || !x_in || !x_out || !xphys_out) { set_error("null argument"); return TOPO_ERR_ARG; }
    GUARD_BEGIN
    Ctx& c = ctx->c;
    if (c.sg.stage) { set_error("a design iteration of this context is still in flight"); return TOPO_ERR_ARG; }
    if (!c.opt_ready) TRET(opt_init(c));
    TCK(cudaMemcpyAsync(c.X.p, x_in, sizeof(double) * c.ne, cudaMemcpyHostToDevice, c.s));
    int rc = opt_step(c);
    TRET(rc);
    TCK(cudaMemcpyAsync(x_out, c.X.p, sizeof(double) * c.ne, cudaMemcpyDeviceToHost, c.s));
    TCK(cudaMemcpyAsync(xphys_out, c.XP.p, sizeof(double) * c.ne, cudaMemcpyDeviceToHost, c.s));
    TCK(cudaStreamSynchronize(c.s));
    if (fx) *fx = c.info.last_fx;
    return rc;
    GUARD_END
}
int topo_opt_vector(topo_ctx* ctx, int which, double** ptr_d) {
    if (!ctx || !ptr_d) { set_error("null argument"); return TOPO_ERR_ARG; }
    Ctx& c = ctx->c;
    TRET(opt_alloc(c));
    double* v[8] = {c.X.p, c.XP.p, c.XF.p, c.Xold.p, c.dfdx.p, c.dgdx.p, c.xmin.p, c.xmax.p};
    if (which < 0 || which > 7) { set_error("vector id out of range"); return TOPO_ERR_ARG; }
    *ptr_d = v[which];
    return 0;
}
int topo_solve_info_get(topo_ctx* ctx, topo_solve_info* info) {
    if (!ctx || !info) { set_error("null argument"); return TOPO_ERR_ARG; }
    Ctx& c = ctx->c;
    c.info.amg_levels = c.nlev;
    for (int l = 0; l < 8; l++) c.info.amg_dofs[l] = l < c.nlev ? c.dl[l].ndof : 0;
    *info = c.info;
    return 0;
}

// ---------------------------------------------------------------- instrumentation
long topo_kernel_launches(void) { return __atomic_load_n(&launch_counter(), __ATOMIC_RELAXED); }

int topo_profile_enable(topo_ctx* ctx, int on) {
    if (!ctx) { set_error("null context"); return TOPO_ERR_ARG; }
    ctx->c.prof.on = on != 0;
    return 0;
}

int topo_profile_read(topo_ctx* ctx, int slot, long* launches, double* total_ms) {
    if (!ctx || !launches || !total_ms || slot < 0 || slot >= PS_COUNT) { set_error("bad argument"); return TOPO_ERR_ARG; }
    Ctx& c = ctx->c;
    GUARD_BEGIN
    TCK(cudaStreamSynchronize(c.s));
    double tot = 0.0;
    for (auto& pr : c.prof.rec[slot]) {
        float ms = 0.f;
        TCK(cudaEventElapsedTime(&ms, pr.first, pr.second));
        tot += ms;
        c.prof.pool.push_back(pr.first);
        c.prof.pool.push_back(pr.second);
    }
    *launches = (long)c.prof.rec[slot].size();
    *total_ms = tot;
    c.prof.rec[slot].clear();
    return 0;
    GUARD_END
}

int topo_amg_level(topo_ctx* ctx, int level, int which, int* nrows, int* ncols, int* bs_r, int* bs_c, long* nnzb,
                   int32_t* rp, int32_t* ci, double* vals) {
    if (!ctx || !nrows || !ncols || !bs_r || !bs_c || !nnzb) { set_error("null argument"); return TOPO_ERR_ARG; }
    GUARD_BEGIN
    std::vector<double> v;
    std::vector<int> r, cc;
    int nr = 0, nc = 0, br = 0, bc = 0;
    TRET(amg_level_copy(ctx->c, level, which, v, r, cc, nr, nc, br, bc));
    *nrows = nr;
    *ncols = nc;
    *bs_r = br;
    *bs_c = bc;
    *nnzb = (long)cc.size();
    if (rp) std::copy(r.begin(), r.end(), rp);
    if (ci) std::copy(cc.begin(), cc.end(), ci);
    if (vals) std::copy(v.begin(), v.end(), vals);
    return 0;
    GUARD_END
}

int topo_graph_aggregate(int n, const int32_t* rp, const int32_t* ci, const unsigned char* excl, int32_t* agg) {
    if (n < 0 || !rp || !ci || !agg) { set_error("bad argument"); return TOPO_ERR_ARG; }
    GUARD_BEGIN
    std::vector<int> r(rp, rp + n + 1), cc(ci, ci + rp[n]), a;
    int na = aggregate_graph(n, r, cc, excl, a);
    std::copy(a.begin(), a.end(), agg);
    return na;
    GUARD_END
}

// ---------------------------------------------------------------- generator + files
int topo_gen_cantilever(int nx, int ny, int nz, int nen, double jitter, uint64_t seed, int load_mode, double* vertex,
                        int32_t* element, int32_t* fixed_dofs, int32_t* load_dofs, double* load_vals, int* n_nodes,
                        int* n_elems, int* n_fixed, int* n_loads) {
    if (nx < 1 || ny < 1 || nz < 1 || (nen != 8 && nen != 4)) { set_error("bad lattice"); return TOPO_ERR_ARG; }
    const long nn = (long)(nx + 1) * (ny + 1) * (nz + 1);
    const long ne = (long)nx * ny * nz * (nen == 8 ? 1 : 6);
    if (nn * 3 >= (1L << 31) || ne * nen >= (1L << 31)) { set_error("lattice too large"); return TOPO_ERR_ARG; }
    if (n_nodes) *n_nodes = (int)nn;
    if (n_elems) *n_elems = (int)ne;
    if (n_fixed) *n_fixed = 3 * (ny + 1) * (nz + 1);
    if (n_loads) *n_loads = load_mode == 0 ? (ny + 1) : (nz + 1);
    if (vertex) {
        uint64_t s = seed;
        long n = 0;
        for (int k = 0; k <= nz; k++)
            for (int j = 0; j <= ny; j++)
                for (int i = 0; i <= nx; i++, n++) {
                    const int idx[3] = {i, j, k};
                    const bool interior = i > 0 && i < nx && j > 0 && j < ny && k > 0 && k < nz;
                    for (int q = 0; q < 3; q++) {
                        double u = sm64_unit(s);
                        double x = (double)idx[q] * 1.0;
                        if (nen == 8 || interior) x = x + (2.0 * u - 1.0) * (jitter * 1.0);
                        vertex[3 * n + q] = x;
                    }
                }
    }
    if (element) {
        static const int path[6][2] = {{1, 3}, {1, 5}, {2, 3}, {2, 6}, {4, 5}, {4, 6}};
        long e = 0;
        for (int k = 0; k < nz; k++)
            for (int j = 0; j < ny; j++)
                for (int i = 0; i < nx; i++) {
                    int hex[8];
                    for (int l = 0; l < 8; l++)
                        hex[l] = (i + (l & 1)) + (nx + 1) * ((j + ((l >> 1) & 1)) + (ny + 1) * (k + ((l >> 2) & 1)));
                    if (nen == 8) {
                        for (int l = 0; l < 8; l++) element[8 * e + l] = hex[l];
                        e++;
                        continue;
                    }
                    if (!vertex) { set_error("tet4 generation needs the vertex buffer"); return TOPO_ERR_ARG; }
                    for (int t = 0; t < 6; t++, e++) {
                        int v[4] = {hex[0], hex[path[t][0]], hex[path[t][1]], hex[7]};
                        double d[3][3];
                        for (int a = 0; a < 3; a++)
                            for (int q = 0; q < 3; q++) d[a][q] = vertex[3L * v[a + 1] + q] - vertex[3L * v[0] + q];
                        double det = d[0][0] * (d[1][1] * d[2][2] - d[1][2] * d[2][1]) -
                                     d[0][1] * (d[1][0] * d[2][2] - d[1][2] * d[2][0]) +
                                     d[0][2] * (d[1][0] * d[2][1] - d[1][1] * d[2][0]);
                        if (det < 0.0) std::swap(v[1], v[2]);
                        for (int q = 0; q < 4; q++) element[4 * e + q] = v[q];
                    }
                }
    }
    if (fixed_dofs) {
        int f = 0;
        for (int k = 0; k <= nz; k++)
            for (int j = 0; j <= ny; j++) {
                int n = (nx + 1) * (j + (ny + 1) * k);
                fixed_dofs[f++] = 3 * n; fixed_dofs[f++] = 3 * n + 1; fixed_dofs[f++] = 3 * n + 2;
            }
    }
    if (load_dofs && load_vals) {
        int q = 0;
        if (load_mode == 0)
            for (int j = 0; j <= ny; j++) {
                int n = nx + (nx + 1) * (j + (ny + 1) * 0);
                load_dofs[q] = 3 * n + 2; load_vals[q] = -1.0 / (double)(ny + 1); q++;
            }
        else
            for (int k = 0; k <= nz; k++) {
                int n = nx + (nx + 1) * (0 + (ny + 1) * k);
                load_dofs[q] = 3 * n + 1; load_vals[q] = 1.0; q++;
            }
    }
    return 0;
}

int topo_gen_multiload(int nx, int ny, int nz, int k, uint64_t seed, int32_t* load_dofs, double* load_vals) {
    if (!load_dofs || !load_vals || k < 1) { set_error("bad argument"); return TOPO_ERR_ARG; }
    uint64_t s = seed;
    for (int c = 0; c < k; c++) {
        int j = (int)(sm64_unit(s) * (double)(ny + 1));
        int kk = (int)(sm64_unit(s) * (double)(nz + 1));
        if (j > ny) j = ny;
        if (kk > nz) kk = nz;
        double zc = 2.0 * sm64_unit(s) - 1.0;
        double ph = 6.283185307179586 * sm64_unit(s);
        double rr = std::sqrt(1.0 - zc * zc);
        double d[3] = {rr * std::cos(ph), rr * std::sin(ph), zc};
        int n = nx + (nx + 1) * (j + (ny + 1) * kk);
        for (int q = 0; q < 3; q++) { load_dofs[3 * c + q] = 3 * n + q; load_vals[3 * c + q] = d[q]; }
    }
    return 0;
}

static bool read_numbers(const std::string& path, std::vector<double>& out) {
    std::ifstream f(path);
    if (!f.is_open()) return false;
    out.clear();
    double v;
    while (f >> v) out.push_back(v);
    return true;
}

int topo_read_mesh_dir(const char* dir, int nen, int n_cases, double* vertex, int32_t* element, int32_t* fixed_dofs,
                       int32_t* case_ptr, int32_t* load_dofs, double* load_vals, int* n_nodes, int* n_elems,
                       int* n_fixed, int* n_loads) {
    if (!dir || (nen != 8 && nen != 4) || n_cases < 1) { set_error("bad argument"); return TOPO_ERR_ARG; }
    GUARD_BEGIN
    std::string d(dir);
    std::vector<double> v, e, f;
    if (!read_numbers(d + "/vertex.txt", v)) { set_error("Can't found document::vertex.txt"); return TOPO_ERR_IO; }
    if (!read_numbers(d + "/element.txt", e)) { set_error("Can't found document::element.txt"); return TOPO_ERR_IO; }
    if (!read_numbers(d + "/fixeddofs.txt", f)) { set_error("Can't found document::fixeddofs.txt"); return TOPO_ERR_IO; }
    if (v.size() % 3 || e.size() % nen) { set_error("vertex/element file sizes are not multiples of 3 / nen"); return TOPO_ERR_IO; }
    std::vector<std::vector<double>> ld(n_cases), lv(n_cases);
    long tot = 0;
    for (int c = 0; c < n_cases; c++) {
        std::string a = d + "/loaddof_" + std::to_string(c + 1) + ".txt", b = d + "/load_" + std::to_string(c + 1) + ".txt";
        if (!read_numbers(a, ld[c]) || !read_numbers(b, lv[c])) { set_error("Can't found document::%s", a.c_str()); return TOPO_ERR_IO; }
        if (ld[c].size() != lv[c].size()) { set_error("load DOF and value counts differ for case %d", c + 1); return TOPO_ERR_IO; }
        tot += (long)ld[c].size();
    }
    if (n_nodes) *n_nodes = (int)(v.size() / 3);
    if (n_elems) *n_elems = (int)(e.size() / nen);
    if (n_fixed) *n_fixed = (int)f.size();
    if (n_loads) *n_loads = (int)tot;
    if (vertex) for (size_t i = 0; i < v.size(); i++) vertex[i] = v[i];
    if (element) for (size_t i = 0; i < e.size(); i++) element[i] = (int32_t)e[i];
    if (fixed_dofs) for (size_t i = 0; i < f.size(); i++) fixed_dofs[i] = (int32_t)f[i];
    if (case_ptr) {
        case_ptr[0] = 0;
        for (int c = 0; c < n_cases; c++) case_ptr[c + 1] = case_ptr[c] + (int32_t)ld[c].size();
    }
    if (load_dofs && load_vals) {
        long q = 0;
        for (int c = 0; c < n_cases; c++)
            for (size_t i = 0; i < ld[c].size(); i++, q++) { load_dofs[q] = (int32_t)ld[c][i]; load_vals[q] = lv[c][i]; }
    }
    return 0;
    GUARD_END
}

int topo_write_vtu(topo_ctx* ctx, const char* dir, int itr, const double* xphys_d) {
    if (!ctx || !dir) { set_error("null argument"); return TOPO_ERR_ARG; }
    GUARD_BEGIN
    Ctx& c = ctx->c;
    std::vector<double> U(c.ndof, 0.0), X(c.ne, 0.0);
    if (c.U.p) TCK(cudaMemcpyAsync(U.data(), c.U.p, sizeof(double) * c.ndof, cudaMemcpyDeviceToHost, c.s));
    const double* xsrc = xphys_d ? xphys_d : c.XP.p;
    if (xsrc) TCK(cudaMemcpyAsync(X.data(), xsrc, sizeof(double) * c.ne, cudaMemcpyDeviceToHost, c.s));
    TCK(cudaStreamSynchronize(c.s));
    std::string name = itr == 0 ? "output_initial" : (itr == -1 ? "output_final" : "output_" + std::to_string(itr));
    std::string path = std::string(dir) + "/" + name + ".vtu";
    FILE* f = fopen(path.c_str(), "w");
    if (!f) { set_error("can't create a new vtu file(%s), please make sure you have write permission", path.c_str()); return TOPO_ERR_IO; }
    fprintf(f, "<?xml version=\"1.0\"?>\n<VTKFile type=\"UnstructuredGrid\" version=\"1.0\">\n<UnstructuredGrid>\n");
    fprintf(f, "<Piece NumberOfPoints=\"%d\" NumberOfCells=\"%d\">\n", c.nn, c.ne);
    fprintf(f, "<Points>\n<DataArray type=\"Float64\" Name=\"nodes\" NumberOfComponents=\"3\" format=\"ascii\">\n");
    for (int i = 0; i < c.nn; i++)
        fprintf(f, "%e %e %e\n", c.vertex_h[3L * i], c.vertex_h[3L * i + 1], c.vertex_h[3L * i + 2]);
    fprintf(f, "</DataArray>\n</Points>\n<Cells>\n<DataArray type=\"Int32\" Name=\"connectivity\" NumberOfComponents=\"1\" format=\"ascii\">\n");
    static const int hexo[8] = {0, 1, 3, 2, 4, 5, 7, 6};  // diagonal -> VTK (Write2Vtu.cpp:87-96)
    for (int e = 0; e < c.ne; e++) {
        for (int l = 0; l < c.nen; l++) {
            int ll = c.nen == 8 ? hexo[l] : l;
            fprintf(f, l + 1 < c.nen ? "%d " : "%d", c.elem_h[(long)e * c.nen + ll]);
        }
        fprintf(f, "\n");
    }
    fprintf(f, "</DataArray>\n<DataArray type=\"Int32\" Name=\"offsets\" NumberOfComponents=\"1\" format=\"ascii\">\n");
    for (int e = 0; e < c.ne; e++) fprintf(f, "%d ", (e + 1) * c.nen);
    fprintf(f, "\n</DataArray>\n<DataArray type=\"Int32\" Name=\"types\" NumberOfComponents=\"1\" format=\"ascii\">\n");
    for (int e = 0; e < c.ne; e++) fprintf(f, "%d ", c.nen == 8 ? 12 : 10);
    fprintf(f, "\n</DataArray>\n</Cells>\n<PointData>\n");
    const char* nm[3] = {"ux", "uy", "uz"};
    for (int q = 0; q < 3; q++) {
        fprintf(f, "<DataArray type=\"Float64\" NumberOfComponents=\"1\" Name=\"%s\" format=\"ascii\">\n", nm[q]);
        for (int i = 0; i < c.nn; i++) fprintf(f, "%e ", U[3L * i + q]);
        fprintf(f, "\n</DataArray>\n");
    }
    fprintf(f, "</PointData>\n<CellData>\n<DataArray type=\"Float64\" NumberOfComponents=\"1\" Name=\"xphys\" format=\"ascii\">\n");
    for (int e = 0; e < c.ne; e++) fprintf(f, "%e ", X[e]);
    fprintf(f, "\n</DataArray>\n</CellData>\n</Piece>\n</UnstructuredGrid>\n</VTKFile>\n");
    fclose(f);
    return 0;
    GUARD_END
}

}  // extern "C"
