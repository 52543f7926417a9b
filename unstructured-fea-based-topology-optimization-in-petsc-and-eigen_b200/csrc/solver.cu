// solver.cu -- Krylov solvers of the design iteration:
//   * FGMRES(restart), right-preconditioned by the AMG V-cycle, for K U = F
//     (replaces KSPFGMRES + PCGAMG, SolveFem.cpp:124-139), FP64 Arnoldi and
//     residuals, FP64 or FP32 V-cycle;
//   * Jacobi-preconditioned CG for the Helmholtz filter (KSPCG + PCJACOBI,
//     PDEFilter.cpp:117-137) with PETSc's preconditioned-norm convergence test.
// All reductions are deterministic two-pass block sums.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "ctx.h"

namespace topo {

int kmatvec64r(Ctx& c, const double* u, double* y, const double* b);

constexpr int kRedBlocks = 1184;  // 8 x 148 SMs: enough warps in flight for the vector sweeps
constexpr int kRedMax = 4736;     // largest reduction grid the autotuner tries

// ----------------------------------------------------------------- reductions
__global__ void k_dot(long n, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ part) {
    __shared__ double sm[32];
    double v[1] = {0.0};
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) v[0] += a[i] * b[i];
    block_sum<1>(v, sm);
    if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}
// out[k] = sum_b part[b*nv + k]; optional sqrt of entry `sqrt_idx`
// one warp per value (launch with 32 * min(nv, 32) threads; more values loop)
__global__ void k_final(int nb, int nv, const double* __restrict__ part, double* __restrict__ out, int sqrt_idx) {
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int k = threadIdx.x >> 5; k < nv; k += nw) {
        double v = 0.0;
        for (int i = lane; i < nb; i += 32) v += part[(long)i * nv + k];
        v = warp_sum(v);
        if (lane == 0) out[k] = (k == sqrt_idx) ? sqrt(v) : v;
    }
}
static inline int final_threads(int nv) { return 32 * std::max(1, std::min(nv, 32)); }

int finalize_sum(Ctx& c, const double* partials, int nparts, int nv, double* out_dev) {
    k_final<<<1, final_threads(nv), 0, c.s>>>(nparts, nv, partials, out_dev, -1), note_launch();
    TCK(cudaGetLastError());
    return 0;
}
int dev_dot(Ctx& c, const double* a, const double* b, long n, double* out_dev) {
    if ((long)c.red.n < kRedBlocks * 40L) TRET(c.red.alloc(std::max<long>(kRedBlocks * 40L, 4096)));
    k_dot<<<kRedBlocks, 256, 0, c.s>>>(n, a, b, c.red.p), note_launch();
    return finalize_sum(c, c.red.p, kRedBlocks, 1, out_dev);
}

// ----------------------------------------------------------------- FGMRES kernels
// The last block of a sweep to finish sums the sweep's per-block partials
// part[k * gridDim.x + b] (k < nv) in a fixed order (a warp per sum, lanes
// striding over the blocks) and writes out[k], so no separate launch is
// needed for the grid-level sum; it then re-arms the counter for the next
// sweep.  Optional sqrt of entry `sqrt_idx`.
__device__ __forceinline__ void last_block_sum(int nv, const double* part, double* out, int sqrt_idx,
                                               unsigned* count, bool* last) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) *last = atomicAdd(count, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!*last) return;
    __threadfence();
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5, nb = gridDim.x;
    for (int k = threadIdx.x >> 5; k < nv; k += nw) {
        double v = 0.0;
        for (int i = lane; i < nb; i += 32) v += __ldcg(part + (long)k * nb + i);
        v = warp_sum(v);
        if (lane == 0) out[k] = (k == sqrt_idx) ? sqrt(v) : v;
    }
    if (threadIdx.x == 0) *count = 0u;
}

// h_j = V_j . w for j < nv (classical Gram-Schmidt: one pass over w).
// Two entries per thread and load (16-byte vectors: the basis rows are
// 16-byte aligned, ld even), U grid strides per loop trip so that small nv
// still keeps several loads in flight, the odd last entry by one thread.
// Warp sums by reduce-scatter, block sums by one thread per j.
template <int NV, int U>
__global__ void __launch_bounds__(256) k_mdot(long n, int nv, const double* __restrict__ V, long ld,
                                              const double* __restrict__ w, double* __restrict__ part,
                                              double* __restrict__ out, unsigned* __restrict__ count) {
    __shared__ double sm[8 * NV];
    __shared__ bool last;
    double acc[NV];
#pragma unroll
    for (int j = 0; j < NV; j++) acc[j] = 0.0;
    const long n2 = n >> 1;
    const double2* w2 = reinterpret_cast<const double2*>(w);
    const long stride = (long)gridDim.x * blockDim.x;
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    for (; i + (U - 1) * stride < n2; i += U * stride) {
        double2 wi[U];
#pragma unroll
        for (int u = 0; u < U; u++) wi[u] = w2[i + u * stride];
#pragma unroll
        for (int j = 0; j < NV; j++)
            if (j < nv) {
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const double2 v = reinterpret_cast<const double2*>(V + j * ld)[i + u * stride];
                    acc[j] += v.x * wi[u].x + v.y * wi[u].y;
                }
            }
    }
    for (; i < n2; i += stride) {
        const double2 wi = w2[i];
#pragma unroll
        for (int j = 0; j < NV; j++)
            if (j < nv) {
                const double2 v = reinterpret_cast<const double2*>(V + j * ld)[i];
                acc[j] += v.x * wi.x + v.y * wi.y;
            }
    }
    if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0)
#pragma unroll
        for (int j = 0; j < NV; j++)
            if (j < nv) acc[j] += V[j * ld + n - 1] * w[n - 1];
    const double r = warp_reduce_scatter<NV>(acc);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane < NV) sm[wid * NV + lane] = r;
    __syncthreads();
    if (threadIdx.x < nv) {
        double s = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) s += sm[q * NV + threadIdx.x];
        part[(long)threadIdx.x * gridDim.x + blockIdx.x] = s;
    }
    last_block_sum(nv, part, out, -1, count, &last);
}
// w -= sum_j h_j V_j ; ||w|| (the last block's sum).  With TD the sweep
// runs from the top of the vectors down: k_mdot's last grid strides read the
// top entries of w and of every V_j just before, so when the nv + 1 vectors
// do not all fit in L2 the first strides here still find the ones k_mdot left
// there.  When they do fit, the ascending order is faster (descending
// addresses stream more slowly from DRAM).
template <int NV, int U, bool TD>
__global__ void __launch_bounds__(256) k_orth(long n, int nv, const double* __restrict__ V, long ld,
                                              const double* __restrict__ h, double* __restrict__ w,
                                              double* __restrict__ part, double* __restrict__ norm_out,
                                              unsigned* __restrict__ count) {
    __shared__ double sm[8];
    __shared__ double hs[NV];
    __shared__ bool last;
    if (threadIdx.x < nv) hs[threadIdx.x] = h[threadIdx.x];
    __syncthreads();
    double s = 0.0;
    const long n2 = n >> 1;
    double2* w2 = reinterpret_cast<double2*>(w);
    const long stride = (long)gridDim.x * blockDim.x;
    // entry pair q(i): i from the bottom up, or mirrored from the top down
    const long qb = TD ? n2 - 1 : 0, qs = TD ? -1 : 1;
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    for (; i + (U - 1) * stride < n2; i += U * stride) {
        double2 wi[U];
#pragma unroll
        for (int u = 0; u < U; u++) wi[u] = w2[qb + qs * (i + u * stride)];
#pragma unroll
        for (int j = 0; j < NV; j++)
            if (j < nv) {
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const double2 vv = reinterpret_cast<const double2*>(V + j * ld)[qb + qs * (i + u * stride)];
                    wi[u].x -= hs[j] * vv.x;
                    wi[u].y -= hs[j] * vv.y;
                }
            }
#pragma unroll
        for (int u = 0; u < U; u++) {
            w2[qb + qs * (i + u * stride)] = wi[u];
            s += wi[u].x * wi[u].x + wi[u].y * wi[u].y;
        }
    }
    for (; i < n2; i += stride) {
        double2 wi = w2[qb + qs * i];
#pragma unroll
        for (int j = 0; j < NV; j++)
            if (j < nv) {
                const double2 vv = reinterpret_cast<const double2*>(V + j * ld)[qb + qs * i];
                wi.x -= hs[j] * vv.x;
                wi.y -= hs[j] * vv.y;
            }
        w2[qb + qs * i] = wi;
        s += wi.x * wi.x + wi.y * wi.y;
    }
    if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
        double wi = w[n - 1];
#pragma unroll
        for (int j = 0; j < NV; j++)
            if (j < nv) wi -= hs[j] * V[j * ld + n - 1];
        w[n - 1] = wi;
        s += wi * wi;
    }
    s = warp_sum(s);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sm[wid] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) t += sm[q];
        part[blockIdx.x] = t;
    }
    last_block_sum(1, part, norm_out, 0, count, &last);
}
__global__ void k_scale_to(long n, const double* __restrict__ w, const double* __restrict__ s, double* __restrict__ v,
                           int invert) {
    const double f = invert ? 1.0 / (*s) : (*s);
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) v[i] = w[i] * f;
}
// x += sum_k y_k Z_k (kd from the argument, or from device memory)
template <class TZ>
__global__ void k_update(long n, int kd, const int* __restrict__ kd_dev, const TZ* __restrict__ Z, long ld,
                         const double* __restrict__ y, double* __restrict__ x) {
    __shared__ double ys[128];
    if (kd_dev) kd = *kd_dev;
    if (threadIdx.x < kd) ys[threadIdx.x] = y[threadIdx.x];
    __syncthreads();
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        double s = x[i];
        for (int k = 0; k < kd; k++) s += ys[k] * (double)Z[k * ld + i];
        x[i] = s;
    }
}

// classical Gram-Schmidt sweeps in chunks of at most 32 basis vectors
// Grid of a grid-stride sweep: the tuned reduction grid, capped at one full
// wave of the kernel (its resident CTAs per SM times the SMs) so that wide
// variants with many accumulators do not run in several rounds.
static int wave_of(const void* kern) {
    int dev = 0, nsm = 148, occ = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 256, 0) != cudaSuccess || occ < 1) occ = 1;
    cudaGetLastError();
    return occ * nsm;
}
template <int NV, int U>
static int mdot_grid(int cap) {
    static const int wave = wave_of(reinterpret_cast<const void*>(k_mdot<NV, U>));
    return std::max(1, std::min(cap, wave));
}
template <int NV, int U, bool TD>
static int orth_grid(int cap) {
    static const int wave = wave_of(reinterpret_cast<const void*>(k_orth<NV, U, TD>));
    return std::max(1, std::min(cap, wave));
}
template <int NV, int U, bool TD>
static void launch_orth(Ctx& c, int g0, long n, int k, const double* Vj, long ld, const double* h, double* w,
                        double* hn_out) {
    k_orth<NV, U, TD><<<orth_grid<NV, U, TD>(g0), 256, 0, c.s>>>(n, k, Vj, ld, h, w, c.red.p, hn_out, c.red_count.p);
}

// out[j] = V_j . w (j < nv), one sweep per 32 basis vectors, each finished by
// its own last block
static int mdot(Ctx& c, int nv, const double* V, long ld, const double* w, double* out) {
    const long n = c.ndof;
    for (int j0 = 0; j0 < nv; j0 += 32) {
        const int k = std::min(32, nv - j0);
        const double* Vj = V + (size_t)j0 * ld;
        const int g0 = c.tune.red_blocks;
        if (k <= 8)
            k_mdot<8, 2><<<mdot_grid<8, 2>(g0), 256, 0, c.s>>>(n, k, Vj, ld, w, c.red.p, out + j0, c.red_count.p);
        else if (k <= 16)
            k_mdot<16, 2><<<mdot_grid<16, 2>(g0), 256, 0, c.s>>>(n, k, Vj, ld, w, c.red.p, out + j0, c.red_count.p);
        else
            k_mdot<32, 1><<<mdot_grid<32, 1>(g0), 256, 0, c.s>>>(n, k, Vj, ld, w, c.red.p, out + j0, c.red_count.p);
        note_launch();
        TCK(cudaGetLastError());
    }
    return 0;
}
static long l2_bytes() {
    static const long b = [] {
        int dev = 0, v = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&v, cudaDevAttrL2CacheSize, dev) != cudaSuccess) { cudaGetLastError(); v = 0; }
        return (long)v;
    }();
    return b;
}
// w -= V h; *hn_out = ||w|| of the fully orthogonalised w (the last sweep's)
static int orth(Ctx& c, int nv, const double* V, long ld, const double* h, double* w, double* hn_out) {
    const long n = c.ndof;
    for (int j0 = 0; j0 < nv; j0 += 32) {
        const int k = std::min(32, nv - j0);
        const double* Vj = V + (size_t)j0 * ld;
        const int g0 = c.tune.red_blocks;
        const bool td = (long)(k + 1) * n * (long)sizeof(double) > l2_bytes();
        if (k <= 8) {
            if (td) launch_orth<8, 2, true>(c, g0, n, k, Vj, ld, h + j0, w, hn_out);
            else launch_orth<8, 2, false>(c, g0, n, k, Vj, ld, h + j0, w, hn_out);
        } else if (k <= 16) {
            if (td) launch_orth<16, 2, true>(c, g0, n, k, Vj, ld, h + j0, w, hn_out);
            else launch_orth<16, 2, false>(c, g0, n, k, Vj, ld, h + j0, w, hn_out);
        } else {
            if (td) launch_orth<32, 1, true>(c, g0, n, k, Vj, ld, h + j0, w, hn_out);
            else launch_orth<32, 1, false>(c, g0, n, k, Vj, ld, h + j0, w, hn_out);
        }
        note_launch();
        TCK(cudaGetLastError());
    }
    return 0;
}

static int precond_apply(Ctx& c, const double* v, int j) {
    const long n = c.ndof;
    cudaEvent_t e0;
    prof_begin(c, PS_VCYCLE, &e0);
    if (c.p.precision == TOPO_PREC_MIXED) TRET(amg_vcycle32(c, v, c.Z32.p + (size_t)j * n));
    else TRET(amg_vcycle64(c, v, c.Z64.p + (size_t)j * n));
    prof_end(c, PS_VCYCLE, e0);
    return 0;
}

// ----------------------------------------------------------------- launch-shape autotuning
// Each candidate shape of a hot kernel is timed (best of 3, CUDA events) on
// this context's own operator and vectors at its first solve; the fastest is
// kept for the context's lifetime.  The timed launches write scratch rows of
// the Krylov basis only.
template <class F>
static int time_best(Ctx& c, F&& fn, double* ms) {
    cudaEvent_t e0, e1;
    TCK(cudaEventCreate(&e0));
    TCK(cudaEventCreate(&e1));
    double best = 1e30;
    for (int rep = 0; rep < 3; rep++) {
        TCK(cudaEventRecord(e0, c.s));
        const int rc = fn();
        TCK(cudaEventRecord(e1, c.s));
        TCK(cudaEventSynchronize(e1));
        float t = 0.f;
        TCK(cudaEventElapsedTime(&t, e0, e1));
        if (rc < 0) { best = 1e30; break; }
        best = std::min(best, (double)t);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = best;
    return 0;
}

int autotune_single(Ctx& c) {
    if (!tuning_on(c) || c.tune.single_done || !c.V.p) return 0;
    c.tune.single_done = true;
    const long n = c.ndof;
    const long ldv = (n + 31) & ~31L;
    double* u = c.V.p;
    double* y = c.V.p + ldv;
    TCK(cudaMemsetAsync(u, 0, sizeof(double) * 2 * ldv, c.s));
    const bool prof = c.prof.on;
    c.prof.on = false;
    double best = 1e30, t = 0.0;
    int pick = c.tune.kmv_block;
    for (int b : {64, 128}) {
        c.tune.kmv_block = b;
        TRET(time_best(c, [&]() { return kmatvec(c, c.Ee64.p, u, y, 1); }, &t));
        if (t < best) { best = t; pick = b; }
    }
    c.tune.kmv_block = pick;
    best = 1e30;
    int pick_v = c.tune.sell_variant;
    pick = c.tune.sell_block;
    for (int sv : {0, 1, 2})
        for (int b : {128, 256}) {
            c.tune.sell_block = b;
            c.tune.sell_variant = sv;
            TRET(time_best(c, [&]() { return amg_level0_apply(c, u, y); }, &t));
            if (t < best) { best = t; pick = b; pick_v = sv; }
        }
    c.tune.sell_block = pick;
    c.tune.sell_variant = pick_v;
    if (c.V.n >= (size_t)17 * ldv) {
        best = 1e30;
        pick = c.tune.red_blocks;
        for (int g : {592, 1184, 2368, 4736}) {
            c.tune.red_blocks = g;
            TRET(time_best(c, [&]() { return mdot(c, 16, c.V.p, ldv, y, c.dsc.p + DS_GM); }, &t));
            if (t < best) { best = t; pick = g; }
        }
        c.tune.red_blocks = pick;
    }
    const int rc = amg_tune_levels(c);
    c.prof.on = prof;
    TRET(rc);
    c.info.tuned[0] = c.tune.kmv_block;
    c.info.tuned[1] = c.tune.sell_block;
    c.info.tuned[2] = c.tune.red_blocks;
    for (int l = 0; l < 8 && l < kMaxLevels; l++) c.info.tuned_lanes[l] = c.tune.bsr_g[l];
    c.info.tuned_lanes[0] = c.tune.sell_variant;  // level 0: row-product shape of the sliced-ELLPACK sweeps
    return 0;
}

// ----------------------------------------------------------------- captured Arnoldi steps
uint64_t sig_mix(uint64_t h, uint64_t v) { return h ^ (v + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2)); }

// Step j of an FGMRES cycle from its CUDA graph.  The graph is captured (on
// a private stream, thread-local mode) the first time step j runs in a solve
// whose buffers match the previous solve's; later solves replay it.  Any
// capture problem turns graphs off for this solver and runs the step
// directly.
int step_graph_run(Ctx& c, StepGraphs& G, int j, bool capture_ok, int (*body)(Ctx&, void*), void* arg) {
    if (!capture_ok || G.disabled || c.prof.on) return body(c, arg);
    if (j < (int)G.exec.size() && G.exec[j]) {
        TCK(cudaGraphLaunch(G.exec[j], c.s));
        __atomic_fetch_add(&launch_counter(), G.launches[j], __ATOMIC_RELAXED);
        return 0;
    }
    if (!G.cap) TCK(cudaStreamCreateWithFlags(&G.cap, cudaStreamNonBlocking));
    cudaStream_t s0 = c.s;
    const long l0 = launch_counter();
    c.s = G.cap;
    cudaError_t e = cudaStreamBeginCapture(G.cap, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        c.s = s0;
        cudaGetLastError();
        G.disabled = true;
        return body(c, arg);
    }
    const int rc = body(c, arg);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(G.cap, &g);
    c.s = s0;
    const long n = launch_counter() - l0;
    cudaGraphExec_t ex = nullptr;
    if (rc >= 0 && e == cudaSuccess && g) e = cudaGraphInstantiate(&ex, g, 0);
    if (g) cudaGraphDestroy(g);
    if (rc < 0 || e != cudaSuccess || !ex) {
        // nothing captured ran: take back its launch count, run directly
        cudaGetLastError();
        __atomic_fetch_sub(&launch_counter(), n, __ATOMIC_RELAXED);
        G.disabled = true;
        return body(c, arg);
    }
    if ((int)G.exec.size() <= j) {
        G.exec.resize(j + 1, nullptr);
        G.launches.resize(j + 1, 0);
    }
    G.exec[j] = ex;
    G.launches[j] = n;
    TCK(cudaGraphLaunch(ex, c.s));  // counted by the capture above
    return 0;
}

// ----------------------------------------------------------------- device-side Arnoldi bookkeeping
// Layout of the per-cycle state (doubles): H (m+1) x m row-major, then cs[m],
// sn[m], g[m+1], y[m].
struct GmLayout {
    int m;
    __host__ __device__ int H(int i, int j) const { return i * m + j; }
    __host__ __device__ int cs(int j) const { return (m + 1) * m + j; }
    __host__ __device__ int sn(int j) const { return (m + 1) * m + m + j; }
    __host__ __device__ int g(int j) const { return (m + 1) * m + 2 * m + j; }
    __host__ __device__ int y(int j) const { return (m + 1) * m + 3 * m + 1 + j; }
    __host__ __device__ int size() const { return (m + 1) * m + 4 * m + 1; }
};

// cycle start: beta = sqrt(||r||^2), g = (beta, 0, ...); beta also to out[0]
__global__ void k_gm_start(GmLayout L, double* __restrict__ st, const double* __restrict__ r2,
                           double* __restrict__ out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double beta = sqrt(*r2);
    for (int j = 0; j <= L.m; j++) st[L.g(j)] = 0.0;
    st[L.g(0)] = beta;
    out[0] = beta;
}
// column j of the Hessenberg matrix (h[0..j] and h[j+1] = ||w||) is rotated
// by the previous Givens rotations, a new rotation zeroes h[j+1,j], and the
// residual estimate |g[j+1]| goes to out[0] (out[1] = ||w||)
__global__ void k_gm_givens(GmLayout L, int j, const double* __restrict__ hcol, double* __restrict__ st,
                            double* __restrict__ out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int i = 0; i <= j + 1; i++) st[L.H(i, j)] = hcol[i];
    for (int i = 0; i < j; i++) {
        const double c = st[L.cs(i)], s = st[L.sn(i)];
        const double t1 = st[L.H(i, j)], t2 = st[L.H(i + 1, j)];
        st[L.H(i, j)] = c * t1 + s * t2;
        st[L.H(i + 1, j)] = -s * t1 + c * t2;
    }
    const double hjj = st[L.H(j, j)], hj1 = st[L.H(j + 1, j)];
    const double den = sqrt(hjj * hjj + hj1 * hj1);
    double c = 1.0, s = 0.0;
    if (den != 0.0) { c = hjj / den; s = hj1 / den; }
    st[L.cs(j)] = c;
    st[L.sn(j)] = s;
    st[L.H(j, j)] = c * hjj + s * hj1;
    st[L.H(j + 1, j)] = 0.0;
    const double gj = st[L.g(j)];
    st[L.g(j + 1)] = -s * gj;
    st[L.g(j)] = c * gj;
    out[0] = fabs(-s * gj);
    out[1] = hcol[j + 1];
}
// y = R^-1 g for the kd completed columns (kd from the argument, or from
// device memory)
__global__ void k_gm_solve(GmLayout L, int kd, const int* __restrict__ kd_dev, double* __restrict__ st) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (kd_dev) kd = *kd_dev;
    for (int i = kd - 1; i >= 0; i--) {
        double s = st[L.g(i)];
        for (int k = i + 1; k < kd; k++) s -= st[L.H(i, k)] * st[L.y(k)];
        st[L.y(i)] = s / st[L.H(i, i)];
    }
}

// Arnoldi step j: z_j = M^-1 v_j, w = K z_j, h = V^T w, w -= V h,
// v_{j+1} = w / ||w||, Givens update, residual estimate to pinned memory.
struct StepArgs {
    int j;
    long n;
    GmLayout GL;
    double *gm, *st, *out, *hs;  // hs: pinned host mirror of out (null: no read-back)
};
static int arnoldi_step(Ctx& c, void* p) {
    const StepArgs& a = *static_cast<const StepArgs*>(p);
    const int j = a.j;
    const long n = a.n;
    const long ldv = (n + 31) & ~31L;  // basis rows 256-byte aligned
    const double* vj = c.V.p + (size_t)j * ldv;
    TRET(precond_apply(c, vj, j));
    if (c.p.precision == TOPO_PREC_MIXED) TRET(kmatvec_f32in(c, c.Ee64.p, c.Z32.p + (size_t)j * n, c.w.p));
    else TRET(kmatvec(c, c.Ee64.p, c.Z64.p + (size_t)j * n, c.w.p));
    cudaEvent_t e0;
    prof_begin(c, PS_ORTH, &e0);
    TRET(mdot(c, j + 1, c.V.p, ldv, c.w.p, a.gm));
    TRET(orth(c, j + 1, c.V.p, ldv, a.gm, c.w.p, a.gm + j + 1));
    prof_end(c, PS_ORTH, e0);
    k_scale_to<<<grid_for(n, 256), 256, 0, c.s>>>(n, c.w.p, a.gm + j + 1, c.V.p + (size_t)(j + 1) * ldv, 1),
        note_launch();
    k_gm_givens<<<1, 32, 0, c.s>>>(a.GL, j, a.gm, a.st, a.out + 2 * j), note_launch();
    if (a.hs) TCK(cudaMemcpyAsync(a.hs + 2 * j, a.out + 2 * j, 2 * sizeof(double), cudaMemcpyDeviceToHost, c.s));
    TCK(cudaGetLastError());
    return 0;
}

// ----------------------------------------------------------------- device-driven FGMRES
// The same FGMRES as fgmres() below, for capture into the step graph
// (stepgraph.cu): the restart cycles are a conditional WHILE node, each
// Arnoldi step j of a cycle an IF node, and single-thread kernels take the
// decisions the host takes in fgmres() (stopping test, restart, iteration
// cap) and set the nodes' conditions.  Every loop is bounded by fem_maxit.
// State in c.di (DiSlot), thresholds in c.dsc.
struct StepHandles {
    cudaGraphConditionalHandle h[128];
    int m;
};
// ttol = max(rtol ||b||, 1e-50); the loop runs while maxit > 0
__global__ void k_dd_init(const double* __restrict__ b2, double rtol, int maxit, int* __restrict__ di,
                          double* __restrict__ ttol, cudaGraphConditionalHandle loop) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    *ttol = fmax(rtol * sqrt(*b2), 1e-50);
    di[DI_ITS] = 0;
    di[DI_CONV] = 0;
    di[DI_STATUS] = 1;
    cudaGraphSetConditional(loop, maxit > 0 ? 1u : 0u);
}
// cycle start: beta = ||b - K x|| already in *beta; converged if beta <= ttol
__global__ void k_dd_cycle(int* __restrict__ di, const double* __restrict__ beta_p, const double* __restrict__ ttol,
                           int maxit, int m, cudaGraphConditionalHandle cyc) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double beta = *beta_p;
    unsigned go = 0;
    if (!isfinite(beta)) di[DI_NAN] = 1;
    else if (beta <= *ttol) di[DI_CONV] = 1;
    else {
        const int jmax = min(m, maxit - di[DI_ITS]);
        di[DI_JMAX] = jmax;
        di[DI_KDONE] = jmax;
        di[DI_STOP] = 0;
        go = jmax > 0;
    }
    cudaGraphSetConditional(cyc, go);
}
// first node of a cycle's body: step 0 runs, steps 1.. wait for their predecessor
__global__ void k_dd_steps_reset(StepHandles H) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int j = 0; j < H.m; j++) cudaGraphSetConditional(H.h[j], j == 0 ? 1u : 0u);
}
// after Arnoldi step j: the check fgmres() does on the host
__global__ void k_dd_step(int j, int* __restrict__ di, const double* __restrict__ out, const double* __restrict__ ttol,
                          cudaGraphConditionalHandle next, int has_next) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double res = out[0], hn = out[1];
    di[DI_ITS] += 1;
    bool stop = false;
    if (!isfinite(res)) {
        di[DI_NAN] = 1;
        di[DI_KDONE] = j + 1;
        stop = true;
    } else if (res <= *ttol || hn == 0.0) {
        di[DI_CONV] = res <= *ttol;
        di[DI_KDONE] = j + 1;
        stop = true;
    }
    if (j + 1 >= di[DI_JMAX]) stop = true;  // the cycle's last step: kdone = jmax
    di[DI_STOP] = stop;
    if (has_next) cudaGraphSetConditional(next, stop ? 0u : 1u);
}
// end of a cycle: restart unless converged, broken down or at the cap
__global__ void k_dd_cycle_end(int* __restrict__ di, int maxit, cudaGraphConditionalHandle loop) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const bool more = !di[DI_CONV] && !di[DI_NAN] && di[DI_ITS] < maxit;
    di[DI_STATUS] = di[DI_CONV] ? 0 : 1;
    cudaGraphSetConditional(loop, more ? 1u : 0u);
}
// ||F - K U|| / ||F|| from the two squared norms
__global__ void k_relres(const double* __restrict__ sq, double* __restrict__ out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    *out = sq[1] > 0 ? sqrt(sq[0] / sq[1]) : sqrt(sq[0]);
}

static int fgmres_dd(Ctx& c, const double* b, double* x) {
    const long n = c.ndof;
    const int m = std::max(1, std::min(c.p.fem_restart, 128));
    const int maxit = c.p.fem_maxit;
    const GmLayout GL{m};
    const long ldv = (n + 31) & ~31L;
    const bool mixed = c.p.precision == TOPO_PREC_MIXED;
    if (!c.V.p || (long)c.V.n < (long)(m + 1) * ldv || (mixed ? !c.Z32.p : !c.Z64.p) ||
        (tuning_on(c) && !c.tune.single_done)) {
        set_error("the device-driven step needs a direct solve of this form first");
        return TOPO_ERR_ARG;
    }
    double* gm = c.dsc.p + DS_GM;
    double* st = c.wtmp.p;
    double* out = st + GL.size();
    double* out_beta = out + 2 * m + 2;
    double* ttol = c.dsc.p + DS_TTOL;
    int* di = c.di.p;
    TRET(dev_dot(c, b, b, n, gm));
    cudaGraphConditionalHandle hloop, hcyc;
    TRET(cond_handle(c, &hloop));
    k_dd_init<<<1, 32, 0, c.s>>>(gm, c.p.fem_rtol, maxit, di, ttol, hloop), note_launch();
    TRET(cond_begin(c, hloop, cudaGraphCondTypeWhile));
    {
        // v0 = (b - K x) / beta
        TRET(kmatvec64r(c, x, c.w.p, b));
        TRET(dev_dot(c, c.w.p, c.w.p, n, gm));
        k_gm_start<<<1, 32, 0, c.s>>>(GL, st, gm, out_beta), note_launch();
        TRET(cond_handle(c, &hcyc));
        k_dd_cycle<<<1, 32, 0, c.s>>>(di, out_beta, ttol, maxit, m, hcyc), note_launch();
        TRET(cond_begin(c, hcyc, cudaGraphCondTypeIf));
        {
            StepHandles H{};
            H.m = m;
            for (int j = 0; j < m; j++) TRET(cond_handle(c, &H.h[j]));
            k_dd_steps_reset<<<1, 32, 0, c.s>>>(H), note_launch();
            k_scale_to<<<grid_for(n, 256), 256, 0, c.s>>>(n, c.w.p, out_beta, c.V.p, 1), note_launch();
            for (int j = 0; j < m; j++) {
                TRET(cond_begin(c, H.h[j], cudaGraphCondTypeIf));
                StepArgs sa{j, n, GL, gm, st, out, nullptr};
                TRET(arnoldi_step(c, &sa));
                k_dd_step<<<1, 32, 0, c.s>>>(j, di, out + 2 * j, ttol, j + 1 < m ? H.h[j + 1] : H.h[j], j + 1 < m),
                    note_launch();
                TRET(cond_end(c));
            }
            k_gm_solve<<<1, 32, 0, c.s>>>(GL, 0, di + DI_KDONE, st), note_launch();
            if (mixed)
                k_update<float><<<grid_for(n, 256), 256, 0, c.s>>>(n, 0, di + DI_KDONE, c.Z32.p, n, st + GL.y(0), x),
                    note_launch();
            else
                k_update<double><<<grid_for(n, 256), 256, 0, c.s>>>(n, 0, di + DI_KDONE, c.Z64.p, n, st + GL.y(0),
                                                                    x), note_launch();
        }
        TRET(cond_end(c));
        k_dd_cycle_end<<<1, 32, 0, c.s>>>(di, maxit, hloop), note_launch();
    }
    TRET(cond_end(c));
    TCK(cudaGetLastError());
    return 0;
}

// FGMRES(restart) on K(Ee64) u = b, x in/out.  Converged when the Arnoldi
// residual estimate |g_{j+1}| <= max(rtol ||b||, 1e-50) (KSPConvergedDefault
// with a nonzero initial guess: rnorm0 = ||b||).  The Hessenberg
// bookkeeping lives on the device and iteration j+1 is queued before the
// host reads iteration j's residual, so the GPU never waits for the host;
// the one speculative iteration of a converged cycle writes only column
// j+1 state and is discarded.
static int fgmres(Ctx& c, const double* b, double* x, int* its_out, int* status) {
    const long n = c.ndof;
    const int m = std::max(1, std::min(c.p.fem_restart, 128));
    const int maxit = c.p.fem_maxit;
    const GmLayout GL{m};
    const long ldv = (n + 31) & ~31L;  // basis rows 256-byte aligned
    if (!c.V.p || (long)c.V.n < (long)(m + 1) * ldv) {
        TRET(c.V.alloc((size_t)(m + 1) * ldv));
        TRET(c.w.alloc(n));
        TRET(c.wtmp.alloc(GL.size() + 2 * m + 8));
        c.Z32.reset();
        c.Z64.reset();
    }
    if (c.p.precision == TOPO_PREC_MIXED && !c.Z32.p) TRET(c.Z32.alloc((size_t)m * n));
    if (c.p.precision != TOPO_PREC_MIXED && !c.Z64.p) TRET(c.Z64.alloc((size_t)m * n));
    if ((long)c.red.n < kRedMax * 40L) TRET(c.red.alloc(std::max<long>(kRedMax * 40L, 4096)));
    while ((int)c.gm_ev.size() < m + 1) {
        cudaEvent_t e;
        TCK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        c.gm_ev.push_back(e);
    }
    TRET(autotune_single(c));
    double* hs = c.hsc.h + 512;     // pinned: [2j, 2j+1] = (residual, ||w||) of iteration j; [300], [301] norms
    double* gm = c.dsc.p + DS_GM;   // Hessenberg column scratch
    double* st = c.wtmp.p;          // device Arnoldi state
    double* out = st + GL.size();   // per-launch outputs (2 doubles per iteration, then beta)
    double* out_beta = out + 2 * m + 2;
    // buffers and options the Arnoldi-step graphs depend on
    uint64_t sig = 0x51ed270b27ull;
    for (uint64_t v : {(uint64_t)(uintptr_t)c.V.p, (uint64_t)(uintptr_t)c.Z32.p, (uint64_t)(uintptr_t)c.Z64.p,
                       (uint64_t)(uintptr_t)c.w.p, (uint64_t)(uintptr_t)c.wtmp.p, (uint64_t)(uintptr_t)c.red.p,
                       (uint64_t)(uintptr_t)c.dsc.p, (uint64_t)(uintptr_t)c.hsc.h, (uint64_t)(uintptr_t)c.Ee64.p,
                       (uint64_t)(uintptr_t)c.v32.A0s.p, (uint64_t)(uintptr_t)c.v64.A0s.p,
                       (uint64_t)(uintptr_t)c.h0.S.p, (uint64_t)c.p.amg_half_fine, (uint64_t)(uintptr_t)c.cinv.p, (uint64_t)(uintptr_t)c.rho.p, (uint64_t)c.p.precision,
                       (uint64_t)m, (uint64_t)c.nlev, (uint64_t)c.p.cheb_degree, (uint64_t)c.p.cheb_degree_post, (uint64_t)c.p.cheb_degree_coarse, (uint64_t)c.p.amg_coarse_cta, (uint64_t)c.p.fine_smoother_matfree, (uint64_t)c.p.pdl,
                       (uint64_t)c.tune.kmv_block, (uint64_t)c.tune.sell_block, (uint64_t)c.tune.red_blocks, (uint64_t)c.tune.sell_variant,
                       (uint64_t)c.tune.bsr_g[1] | (uint64_t)c.tune.bsr_g[2] << 8 | (uint64_t)c.tune.bsr_g[3] << 16 |
                           (uint64_t)c.tune.bsr_g[4] << 24,
                       (uint64_t)n})
        sig = sig_mix(sig, v);
    StepGraphs& G = c.graphs;
    if (G.sig != sig) {
        G.drop();
        G.sig = sig;
    }
    const bool capture_ok = c.p.fem_graphs && G.seen == sig;
    G.seen = sig;
    TRET(dev_dot(c, b, b, n, gm));
    TCK(cudaMemcpyAsync(hs + 300, gm, sizeof(double), cudaMemcpyDeviceToHost, c.s));
    TCK(cudaStreamSynchronize(c.s));
    const double bnorm = std::sqrt(hs[300]);
    const double ttol = std::max(c.p.fem_rtol * bnorm, 1e-50);
    int its = 0;
    bool conv = false;
    cudaEvent_t esolve;
    prof_begin(c, PS_SOLVE, &esolve);
    while (!conv && its < maxit) {
        // v0 = (b - K x) / beta
        TRET(kmatvec64r(c, x, c.w.p, b));
        TRET(dev_dot(c, c.w.p, c.w.p, n, gm));
        k_gm_start<<<1, 32, 0, c.s>>>(GL, st, gm, out_beta), note_launch();
        TCK(cudaMemcpyAsync(hs + 301, out_beta, sizeof(double), cudaMemcpyDeviceToHost, c.s));
        TCK(cudaStreamSynchronize(c.s));
        const double beta = hs[301];
        if (!std::isfinite(beta)) { set_error("FGMRES residual is not finite"); return TOPO_ERR_NAN; }
        if (beta <= ttol) { conv = true; break; }
        k_scale_to<<<grid_for(n, 256), 256, 0, c.s>>>(n, c.w.p, out_beta, c.V.p, 1), note_launch();
        const int jmax = std::min(m, maxit - its);
        int kdone = jmax;
        bool stop = false;
        for (int j = 0; j <= jmax && !stop; j++) {
            if (j < jmax) {
                StepArgs sa{j, n, GL, gm, st, out, hs};
                TRET(step_graph_run(c, G, j, capture_ok, arnoldi_step, &sa));
                TCK(cudaEventRecord(c.gm_ev[j], c.s));
            }
            if (j == 0) continue;
            // check iteration j-1 while iteration j runs
            TCK(cudaEventSynchronize(c.gm_ev[j - 1]));
            its++;
            const double res = hs[2 * (j - 1)], hn = hs[2 * (j - 1) + 1];
            if (!std::isfinite(res)) { set_error("FGMRES breakdown (non-finite residual)"); return TOPO_ERR_NAN; }
            if (res <= ttol || hn == 0.0) {
                conv = res <= ttol;
                kdone = j;
                stop = true;
            }
        }
        k_gm_solve<<<1, 32, 0, c.s>>>(GL, kdone, nullptr, st), note_launch();
        if (c.p.precision == TOPO_PREC_MIXED)
            k_update<float><<<grid_for(n, 256), 256, 0, c.s>>>(n, kdone, nullptr, c.Z32.p, n, st + GL.y(0), x),
                note_launch();
        else
            k_update<double><<<grid_for(n, 256), 256, 0, c.s>>>(n, kdone, nullptr, c.Z64.p, n, st + GL.y(0), x),
                note_launch();
        TCK(cudaGetLastError());
    }
    prof_end(c, PS_SOLVE, esolve);
    *its_out = its;
    *status = conv ? 0 : 1;
    return 0;
}

static int fem_solve_impl(Ctx& c, const double* xphys, double* u);

// SolveFem::ComputeFem (SolveFem.cpp:91-157).  A non-finite density (or any
// breakdown) leaves NaNs in the warm-started spectral estimates and in U; they
// are reset here so that the context stays usable after the error.
int fem_solve(Ctx& c, const double* xphys, double* u) {
    const int rc = fem_solve_impl(c, xphys, u);
    if (rc < 0) {
        c.u_valid = false;
        c.blk.u_valid = c.blk.u_fresh = false;
        amg_reset_warm_start(c);
    }
    return rc;
}

// moduli, AMG numeric setup, U = 0, FGMRES, then the true relative residual
static int fem_solve_impl(Ctx& c, const double* xphys, double* u) {
    if (block_cases(c)) return fem_solve_block(c, xphys, u);
    if (c.sg.dd && c.ncases != 1) {
        set_error("the device-driven step supports one load case (or the block solver)");
        return TOPO_ERR_UNSUPPORTED;
    }
    c.blk.u_valid = c.blk.u_fresh = false;
    TRET(compute_moduli(c, xphys));
    TRET(amg_numeric(c));
    const long n = c.ndof;
    int worst = 0, its_total = 0;
    double rel_worst = 0.0;
    for (int k = 0; k < c.ncases; k++) {
        double* uk = u + (size_t)k * n;
        const double* fk = c.F.p + (size_t)k * n;
        // AssembleFem zeroes U (SolveFem.cpp:333); the optional warm start keeps
        // the previous solution of this context as the initial guess
        if (!(c.p.fem_warm_start && c.u_valid && uk == c.U.p + (size_t)k * n))
            TCK(cudaMemsetAsync(uk, 0, sizeof(double) * n, c.s));
        int its = 0, st = 0;
        if (c.sg.dd) TRET(fgmres_dd(c, fk, uk));
        else TRET(fgmres(c, fk, uk, &its, &st));
        its_total += its;
        worst = std::max(worst, st);
        // true residual ||F - K U|| / ||F||
        TRET(kmatvec64r(c, uk, c.w.p, fk));
        double* gm = c.dsc.p + DS_GM;
        TRET(dev_dot(c, c.w.p, c.w.p, n, gm));
        TRET(dev_dot(c, fk, fk, n, gm + 1));
        if (c.sg.dd) {  // read with the step's other results
            k_relres<<<1, 32, 0, c.s>>>(gm, c.dsc.p + DS_RELRES), note_launch();
            TCK(cudaGetLastError());
            continue;
        }
        TCK(cudaMemcpyAsync(c.hsc.h, gm, 2 * sizeof(double), cudaMemcpyDeviceToHost, c.s));
        TCK(cudaStreamSynchronize(c.s));
        double rel = c.hsc.h[1] > 0 ? std::sqrt(c.hsc.h[0] / c.hsc.h[1]) : std::sqrt(c.hsc.h[0]);
        rel_worst = std::max(rel_worst, rel);
        if (c.p.verbose) printf("Norm of error %e, Iterations %d\n", rel, its);
    }
    c.u_valid = (u == c.U.p);
    if (c.sg.dd) return 0;  // counts and status come from the device after the step
    c.info.fem_its = its_total;
    c.info.fem_relres = rel_worst;
    c.info.fem_status = worst;
    return worst ? TOPO_NOT_CONVERGED : 0;
}

// ----------------------------------------------------------------- filter CG
__global__ void k_cg_start(long n, const double* __restrict__ b, const double* __restrict__ w,
                           const double* __restrict__ dinv, double* __restrict__ r, double* __restrict__ z,
                           double* __restrict__ part) {
    __shared__ double sm[3 * 32];
    double v[3] = {0.0, 0.0, 0.0};
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        double ri = b[i] - w[i], zi = dinv[i] * ri, zb = dinv[i] * b[i];
        r[i] = ri;
        z[i] = zi;
        v[0] += zi * zi;
        v[1] += zi * ri;
        v[2] += zb * zb;
    }
    block_sum<3>(v, sm);
    if (threadIdx.x == 0) for (int k = 0; k < 3; k++) part[3L * blockIdx.x + k] = v[k];
}
// p = z (first) or p = z + (beta/betaold) p; first from the argument, or
// (its_dev) when no iteration has been done yet
__global__ void k_cg_p(long n, const double* __restrict__ z, double* __restrict__ p, const double* __restrict__ sc,
                       int first, const int* __restrict__ its_dev) {
    if (its_dev) first = *its_dev == 0;
    const double bb = first ? 0.0 : sc[2] / sc[3];
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        p[i] = first ? z[i] : z[i] + bb * p[i];
}
// sc[4] = dpi = p.w, the grid sum finished by the last block
__global__ void k_cg_dot(long n, const double* __restrict__ p, const double* __restrict__ w, double* __restrict__ sc,
                         double* __restrict__ part, unsigned* __restrict__ count) {
    __shared__ double sm[32];
    __shared__ bool last;
    double v[1] = {0.0};
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) v[0] += p[i] * w[i];
    block_sum<1>(v, sm);
    if (threadIdx.x == 0) part[blockIdx.x] = v[0];
    last_block_sum(1, part, sc + 4, -1, count, &last);
}
// a = beta/dpi; x += a p; r -= a w; z = Dinv r; then, in the last block to
// finish (every block has read sc by then): sc[1] = dp = sqrt(z.z),
// sc[3] = betaold = sc[2], sc[2] = beta = z.r
__global__ void k_cg_step(long n, const double* __restrict__ p, const double* __restrict__ w,
                          const double* __restrict__ dinv, double* __restrict__ x, double* __restrict__ r,
                          double* __restrict__ z, double* __restrict__ sc, double* __restrict__ part,
                          unsigned* __restrict__ count) {
    __shared__ double sm[2 * 32];
    __shared__ double tot[2];
    __shared__ bool last;
    const double a = sc[2] / sc[4];
    double v[2] = {0.0, 0.0};
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        x[i] += a * p[i];
        double ri = r[i] - a * w[i];
        r[i] = ri;
        double zi = dinv[i] * ri;
        z[i] = zi;
        v[0] += zi * zi;
        v[1] += zi * ri;
    }
    block_sum<2>(v, sm);
    const long nb = gridDim.x;
    if (threadIdx.x == 0) { part[blockIdx.x] = v[0]; part[nb + blockIdx.x] = v[1]; }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(count, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (wid < 2) {
        double t = 0.0;
        for (long i = lane; i < nb; i += 32) t += __ldcg(part + wid * nb + i);
        t = warp_sum(t);
        if (lane == 0) tot[wid] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        sc[1] = sqrt(tot[0]);
        sc[3] = sc[2];
        sc[2] = tot[1];
        *count = 0u;
    }
}
// sc[1] = dp = sqrt(z.z); sc[3] = betaold = sc[2]; sc[2] = beta = z.r (+ sc[0] = snorm on start)
__global__ void k_cg_final(int nb, int nv, const double* __restrict__ part, double* __restrict__ sc, int start) {
    __shared__ double sm[3 * 32];
    double v[3] = {0.0, 0.0, 0.0};
    for (int i = threadIdx.x; i < nb; i += blockDim.x)
        for (int k = 0; k < nv; k++) v[k] += part[(long)i * nv + k];
    block_sum<3>(v, sm);
    if (threadIdx.x == 0) {
        sc[1] = sqrt(v[0]);
        sc[3] = start ? 0.0 : sc[2];
        sc[2] = v[1];
        if (start) sc[0] = sqrt(v[2]);
    }
}

// device-driven CG (for the step graph): the iterations are a conditional
// WHILE node; these kernels take filter_cg()'s host decisions
__global__ void k_cgdd_init(const double* __restrict__ sc, double rtol, double atol, int maxit, int* __restrict__ di,
                            int slot, double* __restrict__ ttol, cudaGraphConditionalHandle loop) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double t = fmax(rtol * sc[0], atol), dp = sc[1];
    *ttol = t;
    di[DI_CG_CUR] = 0;
    di[DI_CG_ITS + slot] = 0;
    di[DI_CG_STATUS + slot] = 0;
    unsigned go = 1;
    if (!isfinite(dp)) { di[DI_NAN] = 1; go = 0; }
    else if (dp <= t) go = 0;
    else if (maxit <= 0) { di[DI_CG_STATUS + slot] = 1; go = 0; }
    else if (sc[2] == 0.0) { di[DI_CG_ITS + slot] = 1; go = 0; }  // beta == 0 before the first step
    cudaGraphSetConditional(loop, go);
}
__global__ void k_cgdd_after(const double* __restrict__ sc, const double* __restrict__ ttol, double dtol, int maxit,
                             int* __restrict__ di, int slot, cudaGraphConditionalHandle loop) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int i = di[DI_CG_CUR] + 1;
    di[DI_CG_CUR] = i;
    di[DI_CG_ITS + slot] = i;
    const double dp = sc[1];
    unsigned go = 1;
    if (!isfinite(dp)) { di[DI_NAN] = 1; go = 0; }
    else if (dp <= *ttol) go = 0;
    else if (dp >= dtol * sc[0]) { di[DI_CG_STATUS + slot] = 1; go = 0; }  // diverged
    else if (i >= maxit) { di[DI_CG_STATUS + slot] = 1; go = 0; }
    else if (sc[2] == 0.0) { di[DI_CG_ITS + slot] = i + 1; go = 0; }
    cudaGraphSetConditional(loop, go);
}

static int filter_cg_dd(Ctx& c, const double* b, double* x, int slot) {
    const long n = c.nn;
    double* sc = c.dsc.p + DS_CG;
    int* di = c.di.p;
    double* ttol = c.dsc.p + DS_CGTOL;
    TRET(filter_kf(c, x, c.fw.p));
    k_cg_start<<<kRedBlocks, 256, 0, c.s>>>(n, b, c.fw.p, c.fdiag_inv.p, c.fr.p, c.fz.p, c.red.p), note_launch();
    k_cg_final<<<1, 512, 0, c.s>>>(kRedBlocks, 3, c.red.p, sc, 1), note_launch();
    cudaGraphConditionalHandle h;
    TRET(cond_handle(c, &h));
    k_cgdd_init<<<1, 32, 0, c.s>>>(sc, c.p.filter_rtol, c.p.filter_atol, c.p.filter_maxit, di, slot, ttol, h),
        note_launch();
    TRET(cond_begin(c, h, cudaGraphCondTypeWhile));
    k_cg_p<<<grid_for(n, 256), 256, 0, c.s>>>(n, c.fz.p, c.fp.p, sc, 0, di + DI_CG_CUR), note_launch();
    TRET(filter_kf(c, c.fp.p, c.fw.p));
    k_cg_dot<<<kRedBlocks, 256, 0, c.s>>>(n, c.fp.p, c.fw.p, sc, c.red.p, c.red_count.p), note_launch();
    k_cg_step<<<kRedBlocks, 256, 0, c.s>>>(n, c.fp.p, c.fw.p, c.fdiag_inv.p, x, c.fr.p, c.fz.p, sc, c.red.p,
                                           c.red_count.p),
        note_launch();
    k_cgdd_after<<<1, 32, 0, c.s>>>(sc, ttol, c.p.filter_dtol, c.p.filter_maxit, di, slot, h), note_launch();
    TRET(cond_end(c));
    TCK(cudaGetLastError());
    return 0;
}

// KSPCG + PCJACOBI with a nonzero initial guess x (PDEFilter.cpp:117-137):
// preconditioned residual norm, converged when ||D^-1 r|| <= max(rtol
// ||D^-1 b||, atol), diverged when it exceeds dtol ||D^-1 b||.  `slot`
// (0..3) names the solve in the device-driven step's counters.
int filter_cg(Ctx& c, const double* b, double* x, int* its_out, int slot) {
    const long n = c.nn;
    double* sc = c.dsc.p + DS_CG;
    double* hs = c.hsc.h + 96;
    if ((long)c.red.n < kRedBlocks * 40L) TRET(c.red.alloc(std::max<long>(kRedBlocks * 40L, 4096)));
    if (c.sg.dd) {
        *its_out = 0;
        return filter_cg_dd(c, b, x, slot);
    }
    TRET(filter_kf(c, x, c.fw.p));
    k_cg_start<<<kRedBlocks, 256, 0, c.s>>>(n, b, c.fw.p, c.fdiag_inv.p, c.fr.p, c.fz.p, c.red.p), note_launch();
    k_cg_final<<<1, 512, 0, c.s>>>(kRedBlocks, 3, c.red.p, sc, 1), note_launch();
    TCK(cudaMemcpyAsync(hs, sc, 5 * sizeof(double), cudaMemcpyDeviceToHost, c.s));
    TCK(cudaStreamSynchronize(c.s));
    const double snorm = hs[0];
    const double ttol = std::max(c.p.filter_rtol * snorm, c.p.filter_atol);
    double dp = hs[1];
    *its_out = 0;
    if (!std::isfinite(dp)) { set_error("filter CG residual is not finite"); return TOPO_ERR_NAN; }
    if (dp <= ttol) return 0;
    int i = 0;
    do {
        *its_out = i + 1;
        if (hs[2] == 0.0) return 0;  // beta == 0
        k_cg_p<<<grid_for(n, 256), 256, 0, c.s>>>(n, c.fz.p, c.fp.p, sc, i == 0, nullptr), note_launch();
        TRET(filter_kf(c, c.fp.p, c.fw.p));
        k_cg_dot<<<kRedBlocks, 256, 0, c.s>>>(n, c.fp.p, c.fw.p, sc, c.red.p, c.red_count.p), note_launch();
        k_cg_step<<<kRedBlocks, 256, 0, c.s>>>(n, c.fp.p, c.fw.p, c.fdiag_inv.p, x, c.fr.p, c.fz.p, sc, c.red.p,
                                               c.red_count.p),
            note_launch();
        TCK(cudaMemcpyAsync(hs, sc, 5 * sizeof(double), cudaMemcpyDeviceToHost, c.s));
        TCK(cudaStreamSynchronize(c.s));
        dp = hs[1];
        if (!std::isfinite(dp)) { set_error("filter CG residual is not finite"); return TOPO_ERR_NAN; }
        if (dp <= ttol) return 0;
        if (dp >= c.p.filter_dtol * snorm) { set_error("filter CG diverged"); return TOPO_NOT_CONVERGED; }
        i++;
    } while (i < c.p.filter_maxit);
    return TOPO_NOT_CONVERGED;
}

}  // namespace topo
