// block_solve.cu -- the k-load displacement solve K(x) [u_1..u_k] = [f_1..f_k]
// for load cases that share one stiffness matrix: FGMRES in lockstep over
// the cases (one Arnoldi process, Hessenberg and stopping test per case, as
// k independent KSPFGMRES solves would have; SolveFem.cpp:124-139), with
// every operator application and preconditioner sweep done once for all
// cases on case-interleaved block vectors (entry (dof, case) at
// dof*KB + case):
//   * the outer operator is the tensor-core block kernel of block.cu;
//   * the AMG V-cycle (the same hierarchy as the single-load path, built once
//     per design iteration) runs on KB right-hand sides at once, so each
//     matrix block is read once for all cases;
//   * the Gram-Schmidt sweeps compute all cases' coefficients in one pass.
// A case that has converged stops contributing (its new basis vectors are
// zero) while the others continue; each case takes its own solution update.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "ctx.h"

namespace topo {

void cheb_coeffs(int deg, double* cr, double* cq);  // amg.cu

// ----------------------------------------------------------------- block V-cycle kernels
// Level-0 operator (sliced ELLPACK) on block vectors.  KB/CPT threads per
// node row, each owning CPT = 16/sizeof(T) consecutive cases, so a
// neighbour's 3 x CPT values are three aligned 16-byte loads and the
// threads of a row read one contiguous 16*KB/CPT-byte run per component;
// the row's matrix blocks are read once per thread group (broadcast).
// MODE 0: y = A x; 1: y = b - A x; 2: Chebyshev step with x = d_old:
// t = A d_old; r -= t; d_new = c1 d_old + c2 Dinv r; xo += d_new.
// The slots of a row are taken in groups of U: the column ids of the next
// group are fetched while the current group's values and neighbour runs are
// gathered (one memory round trip per group instead of two), and with U > 1
// all of a group's loads are issued before its arithmetic.  U (1 or 3) is
// picked by the autotuner: U = 3 holds more registers.
template <class T, int KB, int MODE, int U>
__global__ void __launch_bounds__(256) k_sell_blk(int nrows, const int* __restrict__ sp, const int* __restrict__ sci,
                                                  const T* __restrict__ S, const T* __restrict__ x, T* __restrict__ y,
                                                  const T* __restrict__ b, T* __restrict__ r, T* __restrict__ xo,
                                                  const T* __restrict__ dinv, const double* __restrict__ rho,
                                                  double cr, double cq) {
    constexpr int CPT = 16 / (int)sizeof(T);       // cases per thread
    constexpr int TPR = KB / CPT;                  // threads per row
    const long tid = blockIdx.x * (long)blockDim.x + threadIdx.x;
    const int i = (int)(tid / TPR), g = (int)(tid % TPR);
    if (i >= nrows) return;
    const int s = i >> 5, lane = i & 31;
    const int b0 = sp[s], w = (sp[s + 1] - b0) >> 5;
    const size_t sb = (size_t)(b0 >> 5);
    const int* cp = sci + b0 + lane;
    const int c0 = g * CPT;
    T acc[3][CPT];
#pragma unroll
    for (int q = 0; q < 3; q++)
#pragma unroll
        for (int c = 0; c < CPT; c++) acc[q][c] = T(0);
    int jn[U];
#pragma unroll
    for (int u = 0; u < U; u++) jn[u] = u < w ? __ldg(cp + 32 * u) : 0;
    for (int k = 0; k < w; k += U) {
        int jc[U];
#pragma unroll
        for (int u = 0; u < U; u++) jc[u] = jn[u];
#pragma unroll
        for (int u = 0; u < U; u++) jn[u] = k + U + u < w ? __ldg(cp + 32 * (k + U + u)) : 0;
        T xv[U][3][CPT], av[U][9];
#pragma unroll
        for (int u = 0; u < U; u++) {
            if (k + u < w) {
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    const uint4 t = __ldg(reinterpret_cast<const uint4*>(x + (3L * jc[u] + d) * KB + c0));
                    memcpy(xv[u][d], &t, 16);
                }
                sell_load9<T>(S, sb + k + u, lane, av[u]);
            } else {
#pragma unroll
                for (int d = 0; d < 3; d++)
#pragma unroll
                    for (int c = 0; c < CPT; c++) xv[u][d][c] = T(0);
#pragma unroll
                for (int e = 0; e < 9; e++) av[u][e] = T(0);
            }
        }
#pragma unroll
        for (int u = 0; u < U; u++)
#pragma unroll
            for (int q = 0; q < 3; q++)
#pragma unroll
                for (int c = 0; c < CPT; c++)
                    acc[q][c] += av[u][3 * q] * xv[u][0][c] + av[u][3 * q + 1] * xv[u][1][c] +
                                 av[u][3 * q + 2] * xv[u][2][c];
    }
#pragma unroll
    for (int q = 0; q < 3; q++) {
        const long o = (3L * i + q) * KB + c0;
        T out[CPT];
        if (MODE == 0) {
#pragma unroll
            for (int c = 0; c < CPT; c++) out[c] = acc[q][c];
            *reinterpret_cast<uint4*>(y + o) = *reinterpret_cast<const uint4*>(out);
        } else if (MODE == 1) {
            const uint4 tb = *reinterpret_cast<const uint4*>(b + o);
            T bv[CPT];
            memcpy(bv, &tb, 16);
#pragma unroll
            for (int c = 0; c < CPT; c++) out[c] = bv[c] - acc[q][c];
            *reinterpret_cast<uint4*>(y + o) = *reinterpret_cast<const uint4*>(out);
        } else {
            const double delta = 0.5 * (*rho);
            const T c2 = T(cq / delta), c1 = T(cr);
            const T di = dinv[3L * i + q];
            T rv[CPT], dv[CPT], xw[CPT];
            uint4 t = *reinterpret_cast<const uint4*>(r + o);
            memcpy(rv, &t, 16);
            t = *reinterpret_cast<const uint4*>(x + o);
            memcpy(dv, &t, 16);
            t = *reinterpret_cast<const uint4*>(xo + o);
            memcpy(xw, &t, 16);
#pragma unroll
            for (int c = 0; c < CPT; c++) {
                rv[c] -= acc[q][c];
                out[c] = c1 * dv[c] + c2 * di * rv[c];
                xw[c] += out[c];
            }
            *reinterpret_cast<uint4*>(r + o) = *reinterpret_cast<const uint4*>(rv);
            *reinterpret_cast<uint4*>(y + o) = *reinterpret_cast<const uint4*>(out);
            *reinterpret_cast<uint4*>(xo + o) = *reinterpret_cast<const uint4*>(xw);
        }
    }
}

// Block-sparse (slot-interleaved BSR) times a block vector (mode 0: y = A x;
// 1: y = b - A x; 2: y += A x) with G lanes per row: lane gl of a row's
// group walks slots gl, gl+G, ..., reads the slot's whole BR x BC block
// (coalesced over the group's consecutive slots) and the neighbour's BC*KB
// values (one contiguous run, 16-byte loads), and keeps all BR*KB sums in
// registers; the group combines them with xor shuffles and writes the row's
// BR*KB outputs as one contiguous run.
template <class T, int BR, int BC, int KB, int G>
__global__ void __launch_bounds__(256) k_bsr_blk_g(int nrows, const int* __restrict__ rp, const int* __restrict__ ci,
                                                   const T* __restrict__ A, const T* __restrict__ x, T* __restrict__ y,
                                                   const T* __restrict__ b, int mode) {
    constexpr int NXV = BC * KB;                   // neighbour run length
    constexpr int VPL = 16 / (int)sizeof(T);       // values per 16-byte load
    const long tid = blockIdx.x * (long)blockDim.x + threadIdx.x;
    const int row = (int)(tid / G), gl = (int)(tid % G);
    const bool active = row < nrows;
    T acc[BR][KB];
#pragma unroll
    for (int q = 0; q < BR; q++)
#pragma unroll
        for (int c = 0; c < KB; c++) acc[q][c] = T(0);
    if (active) {
        const int r0 = rp[row], nb = rp[row + 1] - r0;
        const T* Ar = A + (size_t)r0 * BR * BC;
        for (int s = gl; s < nb; s += G) {
            const int j = __ldg(ci + r0 + s);
            const uint4* xq = reinterpret_cast<const uint4*>(x + (size_t)j * NXV);
#pragma unroll
            for (int d = 0; d < BC; d++) {
                T xv[KB];
#pragma unroll
                for (int h = 0; h < KB / VPL; h++) {
                    const uint4 t = __ldg(xq + (d * KB) / VPL + h);
                    memcpy(xv + h * VPL, &t, 16);
                }
#pragma unroll
                for (int q = 0; q < BR; q++) {
                    const T av = __ldg(Ar + (size_t)(q * BC + d) * nb + s);
#pragma unroll
                    for (int c = 0; c < KB; c++) acc[q][c] += av * xv[c];
                }
            }
        }
    }
#pragma unroll
    for (int q = 0; q < BR; q++)
#pragma unroll
        for (int c = 0; c < KB; c++)
#pragma unroll
            for (int o = G / 2; o > 0; o >>= 1) acc[q][c] += __shfl_xor_sync(0xffffffffu, acc[q][c], o);
    if (!active) return;
    T* yr = y + (size_t)row * BR * KB;
    const T* br = b ? b + (size_t)row * BR * KB : nullptr;
#pragma unroll
    for (int q = 0; q < BR; q++)
#pragma unroll
        for (int c = 0; c < KB; c++) {
            const int v = q * KB + c;
            if (v % G != gl) continue;
            if (mode == 0) yr[v] = acc[q][c];
            else if (mode == 1) yr[v] = br[v] - acc[q][c];
            else yr[v] += acc[q][c];
        }
}

// first Chebyshev step on a block vector (the block form of k_cheb_first)
template <class T, int KB>
__global__ void k_cheb_first_blk(long n, const T* __restrict__ b, T* __restrict__ r, T* __restrict__ d,
                                 T* __restrict__ x, const T* __restrict__ dinv, const double* __restrict__ rho,
                                 int zero_init) {
    const double theta = 0.6 * (*rho);
    const T it = T(1.0 / theta);
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n * KB; i += (long)gridDim.x * blockDim.x) {
        const T di = dinv[i / KB];
        if (zero_init) {
            const T bi = b[i];
            r[i] = bi;
            const T v = di * bi * it;
            d[i] = v;
            x[i] = v;
        } else {
            const T v = di * r[i] * it;
            d[i] = v;
            x[i] += v;
        }
    }
}
template <class T, int KB>
__global__ void k_cheb_upd_blk(long n, const T* __restrict__ t, T* __restrict__ r, const T* __restrict__ dold,
                               T* __restrict__ dnew, T* __restrict__ x, const T* __restrict__ dinv,
                               const double* __restrict__ rho, double cr, double cq) {
    const double delta = 0.5 * (*rho);
    const T c2 = T(cq / delta), c1 = T(cr);
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n * KB; i += (long)gridDim.x * blockDim.x) {
        const T rn = r[i] - t[i];
        const T dn = c1 * dold[i] + c2 * dinv[i / KB] * rn;
        r[i] = rn;
        dnew[i] = dn;
        x[i] += dn;
    }
}
// coarsest level: x = inv b (dense FP64 inverse, n <= a few hundred)
template <class T, int KB>
__global__ void k_dense_apply_blk(int n, const double* __restrict__ inv, const T* __restrict__ b, T* __restrict__ x) {
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = gid / KB, c = gid % KB;
    if (i >= n) return;
    double s = 0.0;
    for (int j = 0; j < n; j++) s += inv[(size_t)i * n + j] * (double)b[(size_t)j * KB + c];
    x[(size_t)i * KB + c] = T(s);
}
template <class TI, class TO>
__global__ void k_convert_blk(long n, const TI* __restrict__ a, TO* __restrict__ b) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) b[i] = (TO)a[i];
}

// ----------------------------------------------------------------- block V-cycle (host)
template <class T>
static AmgVals<T>& avals(Ctx& c);
template <>
AmgVals<double>& avals<double>(Ctx& c) { return c.v64; }
template <>
AmgVals<float>& avals<float>(Ctx& c) { return c.v32; }
template <class T>
static AmgBlkVecs<T>& bvecs(Ctx& c);
template <>
AmgBlkVecs<double>& bvecs<double>(Ctx& c) { return c.blk.bv64; }
template <>
AmgBlkVecs<float>& bvecs<float>(Ctx& c) { return c.blk.bv32; }

template <class T>
static int alloc_bvecs(Ctx& c) {
    AmgBlkVecs<T>& v = bvecs<T>(c);
    if (v.kb == c.blk.kb && v.nlev == c.nlev) return 0;
    const int kb = c.blk.kb;
    for (int l = 0; l < c.nlev; l++) {
        const size_t n = (size_t)c.dl[l].ndof * kb;
        TRET(v.x[l].alloc(n));
        TRET(v.b[l].alloc(n));
        TRET(v.r[l].alloc(n));
        TRET(v.d[l].alloc(n));
        TRET(v.d2[l].alloc(n));
        TRET(v.t[l].alloc(n));
    }
    v.kb = kb;
    v.nlev = c.nlev;
    return 0;
}

template <class T, int BR, int BC, int KB, int G>
static void bsr_launch(Ctx& c, const DevPattern& P, const T* A, const T* x, T* y, const T* b, int mode) {
    const long nt = (long)P.nrows * G;
    k_bsr_blk_g<T, BR, BC, KB, G><<<(int)((nt + 255) / 256), 256, 0, c.s>>>(P.nrows, P.rp.p, P.ci.p, A, x, y, b, mode);
}
template <class T, int BR, int BC, int KB>
static void bsr_launch_g(Ctx& c, const DevPattern& P, const T* A, const T* x, T* y, const T* b, int mode) {
    const double avg = P.nrows ? (double)P.nnzb / P.nrows : 1.0;
    if (avg >= 24.0) bsr_launch<T, BR, BC, KB, 32>(c, P, A, x, y, b, mode);
    else if (avg >= 12.0) bsr_launch<T, BR, BC, KB, 16>(c, P, A, x, y, b, mode);
    else if (avg >= 6.0) bsr_launch<T, BR, BC, KB, 8>(c, P, A, x, y, b, mode);
    else bsr_launch<T, BR, BC, KB, 4>(c, P, A, x, y, b, mode);
}
template <class T, int KB>
static int bsr_apply(Ctx& c, const DevPattern& P, const T* A, int br, int bc, const T* x, T* y, const T* b, int mode) {
    if (br == 3 && bc == 3) bsr_launch_g<T, 3, 3, KB>(c, P, A, x, y, b, mode);
    else if (br == 3 && bc == 6) bsr_launch_g<T, 3, 6, KB>(c, P, A, x, y, b, mode);
    else if (br == 6 && bc == 3) bsr_launch_g<T, 6, 3, KB>(c, P, A, x, y, b, mode);
    else bsr_launch_g<T, 6, 6, KB>(c, P, A, x, y, b, mode);
    note_launch();
    TCK(cudaGetLastError());
    return 0;
}

template <class T, int KB>
static int sell_grid(int nrows) {
    const long nt = (long)nrows * (KB / (16 / (int)sizeof(T)));
    return (int)((nt + 255) / 256);
}

// level-0 block sweep in the slot-group form picked by the autotuner
template <class T, int KB, int MODE>
static void launch_sell_blk(Ctx& c, const T* x, T* y, const T* b, T* r, T* xo, const T* dinv, const double* rho,
                            double cr, double cq) {
    const AmgDevLevel& D = c.dl[0];
    const T* S = avals<T>(c).A0s.p;
    const int grid = sell_grid<T, KB>(D.nnode);
    if (c.tune.blk_sell_u == 3)
        k_sell_blk<T, KB, MODE, 3><<<grid, 256, 0, c.s>>>(D.nnode, D.sell_ptr.p, D.sell_ci.p, S, x, y, b, r, xo,
                                                          dinv, rho, cr, cq);
    else
        k_sell_blk<T, KB, MODE, 1><<<grid, 256, 0, c.s>>>(D.nnode, D.sell_ptr.p, D.sell_ci.p, S, x, y, b, r, xo,
                                                          dinv, rho, cr, cq);
    note_launch();
}

// level operator on block vectors: mode 0 y = A x, 1 y = b - A x
template <class T, int KB>
static int level_apply(Ctx& c, int l, const T* x, T* y, const T* b, int mode) {
    AmgVals<T>& v = avals<T>(c);
    const AmgDevLevel& D = c.dl[l];
    if (l == 0) {
        cudaEvent_t e0;
        const bool rec = mode == 1;
        if (rec) prof_begin(c, PS_RES0, &e0);
        if (mode == 0) launch_sell_blk<T, KB, 0>(c, x, y, b, nullptr, nullptr, nullptr, nullptr, 0, 0);
        else launch_sell_blk<T, KB, 1>(c, x, y, b, nullptr, nullptr, nullptr, nullptr, 0, 0);
        if (rec) prof_end(c, PS_RES0, e0);
        TCK(cudaGetLastError());
        return 0;
    }
    return bsr_apply<T, KB>(c, D.A, v.A[l].p, D.bs, D.bs, x, y, b, mode);
}

template <class T, int KB>
static int smooth_blk(Ctx& c, int l, const T* b, T* x, bool zero_init) {
    AmgVals<T>& v = avals<T>(c);
    AmgBlkVecs<T>& w = bvecs<T>(c);
    const AmgDevLevel& D = c.dl[l];
    const long n = D.ndof;
    int deg = (!zero_init && c.p.cheb_degree_post > 0) ? c.p.cheb_degree_post : c.p.cheb_degree;
    if (l > 0 && c.p.cheb_degree_coarse > 0) deg = c.p.cheb_degree_coarse;
    deg = std::max(1, std::min(deg, 16));
    double cr[16] = {0}, cq[16] = {0};
    cheb_coeffs(deg, cr, cq);
    const double* rho = c.rho.p + 2 * kMaxLevels + l;
    if (!zero_init) TRET((level_apply<T, KB>(c, l, x, w.r[l].p, b, 1)));
    k_cheb_first_blk<T, KB><<<grid_for(n * KB, 256), 256, 0, c.s>>>(n, b, w.r[l].p, w.d[l].p, x, v.dinv[l].p, rho,
                                                                     zero_init ? 1 : 0), note_launch();
    T* dcur = w.d[l].p;
    T* dnxt = w.d2[l].p;
    for (int k = 1; k < deg; k++) {
        if (l == 0) {
            cudaEvent_t e0;
            prof_begin(c, PS_CHEB0, &e0);
            launch_sell_blk<T, KB, 2>(c, dcur, dnxt, nullptr, w.r[l].p, x, v.dinv[l].p, rho, cr[k], cq[k]);
            prof_end(c, PS_CHEB0, e0);
        } else {
            TRET((level_apply<T, KB>(c, l, dcur, w.t[l].p, nullptr, 0)));
            k_cheb_upd_blk<T, KB><<<grid_for(n * KB, 256), 256, 0, c.s>>>(n, w.t[l].p, w.r[l].p, dcur, dnxt, x,
                                                                           v.dinv[l].p, rho, cr[k], cq[k]), note_launch();
        }
        std::swap(dcur, dnxt);
        TCK(cudaGetLastError());
    }
    return 0;
}

template <class T, int KB>
static int vcycle_blk(Ctx& c, const T* b0, T* x0) {
    AmgVals<T>& v = avals<T>(c);
    AmgBlkVecs<T>& w = bvecs<T>(c);
    const int L = c.nlev - 1;
    const T* bl[kMaxLevels];
    T* xl[kMaxLevels];
    for (int l = 0; l <= L; l++) { bl[l] = w.b[l].p; xl[l] = w.x[l].p; }
    bl[0] = b0;
    xl[0] = x0;
    for (int l = 0; l < L; l++) {
        const AmgDevLevel& D = c.dl[l];
        TRET((smooth_blk<T, KB>(c, l, bl[l], xl[l], true)));
        TRET((level_apply<T, KB>(c, l, xl[l], w.t[l].p, bl[l], 1)));
        TRET((bsr_apply<T, KB>(c, D.R, v.R[l].p, 6, D.bs, w.t[l].p, w.b[l + 1].p, nullptr, 0)));
    }
    {
        const int n = c.dl[L].ndof;
        k_dense_apply_blk<T, KB><<<(n * KB + 127) / 128, 128, 0, c.s>>>(n, c.cinv.p, w.b[L].p, w.x[L].p), note_launch();
        TCK(cudaGetLastError());
    }
    for (int l = L - 1; l >= 0; l--) {
        const AmgDevLevel& D = c.dl[l];
        TRET((bsr_apply<T, KB>(c, D.P, v.P[l].p, D.bs, 6, w.x[l + 1].p, xl[l], nullptr, 2)));
        TRET((smooth_blk<T, KB>(c, l, bl[l], xl[l], false)));
    }
    return 0;
}

template <class T>
static int vcycle_blk_any(Ctx& c, const T* b0, T* x0) {
    if (c.blk.kb == 4) return vcycle_blk<T, 4>(c, b0, x0);
    if (c.blk.kb == 8) return vcycle_blk<T, 8>(c, b0, x0);
    return vcycle_blk<T, 16>(c, b0, x0);
}

// z = M^-1 v on block vectors (FP64 in; FP32 or FP64 out)
static int precond_blk(Ctx& c, const double* v, int j) {
    const long nf = (long)c.ndof * c.blk.kb;
    if (c.p.precision == TOPO_PREC_MIXED) {
        TRET(alloc_bvecs<float>(c));
        float* b0 = c.blk.bv32.b[0].p;
        k_convert_blk<double, float><<<grid_for(nf, 256), 256, 0, c.s>>>(nf, v, b0), note_launch();
        TCK(cudaGetLastError());
        return vcycle_blk_any<float>(c, b0, c.blk.Z32.p + (size_t)j * nf);
    }
    TRET(alloc_bvecs<double>(c));
    return vcycle_blk_any<double>(c, v, c.blk.Z64.p + (size_t)j * nf);
}

// ----------------------------------------------------------------- block Krylov kernels
// Per-case reductions over a block vector of n*KB entries: a thread keeps
// one case (its stride is a multiple of KB), lanes of equal case combine by
// xor shuffles of offsets >= KB, warps through shared memory.
template <int KB>
__device__ __forceinline__ double case_warp_sum(double v) {
#pragma unroll
    for (int o = 16; o >= KB; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// part[blk][j][case] = sum_i V_j[i] w[i] over this block's entries.  Two
// consecutive entries (cases c, c+1) per thread and 16-byte load; lanes
// with the same case pair combine by xor shuffles of offsets >= KB/2.
template <int KB>
__device__ __forceinline__ double case2_warp_sum(double v) {
#pragma unroll
    for (int o = 16; o >= KB / 2; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
template <int NV, int KB>
__global__ void __launch_bounds__(256) k_mdot_blk(long nf, int nv, const double* __restrict__ V, long ld,
                                                  const double* __restrict__ w, double* __restrict__ part) {
    __shared__ double sm[8][NV * KB];
    double acc[NV][2];
#pragma unroll
    for (int j = 0; j < NV; j++) acc[j][0] = acc[j][1] = 0.0;
    const long n2 = nf >> 1;
    const double2* w2 = reinterpret_cast<const double2*>(w);
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n2; i += (long)gridDim.x * blockDim.x) {
        const double2 wi = w2[i];
#pragma unroll
        for (int j = 0; j < NV; j++)
            if (j < nv) {
                const double2 v = reinterpret_cast<const double2*>(V + j * ld)[i];
                acc[j][0] += v.x * wi.x;
                acc[j][1] += v.y * wi.y;
            }
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int c0 = (2 * lane) % KB;
#pragma unroll
    for (int j = 0; j < NV; j++) {
        const double s0 = case2_warp_sum<KB>(acc[j][0]), s1 = case2_warp_sum<KB>(acc[j][1]);
        if (lane < KB / 2 && j < nv) {
            sm[wid][j * KB + c0] = s0;
            sm[wid][j * KB + c0 + 1] = s1;
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < nv * KB; t += blockDim.x) {
        double s = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) s += sm[q][t];
        part[(long)blockIdx.x * nv * KB + t] = s;
    }
}
// w -= sum_j h[j][case] V_j ; part[blk][case] = partial ||w_case||^2
template <int NV, int KB>
__global__ void __launch_bounds__(256) k_orth_blk(long nf, int nv, const double* __restrict__ V, long ld,
                                                  const double* __restrict__ h, double* __restrict__ w,
                                                  double* __restrict__ part) {
    __shared__ double hs[NV * KB];
    __shared__ double sm[8][KB];
    for (int t = threadIdx.x; t < nv * KB; t += blockDim.x) hs[t] = h[t];
    __syncthreads();
    const int c0 = (2 * threadIdx.x) % KB;
    double n0 = 0.0, n1 = 0.0;
    const long n2 = nf >> 1;
    double2* w2 = reinterpret_cast<double2*>(w);
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n2; i += (long)gridDim.x * blockDim.x) {
        double2 wi = w2[i];
#pragma unroll
        for (int j = 0; j < NV; j++)
            if (j < nv) {
                const double2 v = reinterpret_cast<const double2*>(V + j * ld)[i];
                wi.x -= hs[j * KB + c0] * v.x;
                wi.y -= hs[j * KB + c0 + 1] * v.y;
            }
        w2[i] = wi;
        n0 += wi.x * wi.x;
        n1 += wi.y * wi.y;
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    n0 = case2_warp_sum<KB>(n0);
    n1 = case2_warp_sum<KB>(n1);
    if (lane < KB / 2) {
        sm[wid][c0] = n0;
        sm[wid][c0 + 1] = n1;
    }
    __syncthreads();
    if (threadIdx.x < KB) {
        double s = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) s += sm[q][threadIdx.x];
        part[(long)blockIdx.x * KB + threadIdx.x] = s;
    }
}
// out[k] = sum_b part[b*nv + k] (sqrt if do_sqrt), one warp per value
__global__ void k_final_blk(int nb, int nv, const double* __restrict__ part, double* __restrict__ out, int do_sqrt) {
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int k = threadIdx.x >> 5; k < nv; k += nw) {
        double v = 0.0;
        for (int i = lane; i < nb; i += 32) v += part[(long)i * nv + k];
        v = warp_sum(v);
        if (lane == 0) out[k] = do_sqrt ? sqrt(v) : v;
    }
}
// v = w / nrm[case] for active cases, 0 otherwise
template <int KB>
__global__ void k_scale_blk(long nf, const double* __restrict__ w, const double* __restrict__ nrm,
                            const int* __restrict__ act, double* __restrict__ v) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < nf; i += (long)gridDim.x * blockDim.x) {
        const int cs = (int)(i % KB);
        const double s = nrm[cs];
        v[i] = (act[cs] && s > 0.0) ? w[i] / s : 0.0;
    }
}
// x += sum_{k < kd_c} y_c[k] Z_k per case
template <class TZ, int KB>
__global__ void k_update_blk(long nf, const TZ* __restrict__ Z, long ld, const double* __restrict__ st, int gsize,
                             int yoff, const int* __restrict__ kd, double* __restrict__ x) {
    __shared__ double ys[KB][129];
    __shared__ int kds[KB];
    if (threadIdx.x < KB) kds[threadIdx.x] = kd[threadIdx.x];
    __syncthreads();
    for (int t = threadIdx.x; t < KB * 128; t += blockDim.x) {
        const int cs = t / 128, k = t % 128;
        ys[cs][k] = k < kds[cs] ? st[(long)cs * gsize + yoff + k] : 0.0;
    }
    __syncthreads();
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < nf; i += (long)gridDim.x * blockDim.x) {
        const int cs = (int)(i % KB);
        double s = x[i];
        const int kdc = kds[cs];
        for (int k = 0; k < kdc; k++) s += ys[cs][k] * (double)Z[k * ld + i];
        x[i] = s;
    }
}

// per-case Arnoldi state: H (m+1) x m, cs[m], sn[m], g[m+1], y[m]
struct GmL {
    int m;
    __host__ __device__ int H(int i, int j) const { return i * m + j; }
    __host__ __device__ int cs(int j) const { return (m + 1) * m + j; }
    __host__ __device__ int sn(int j) const { return (m + 1) * m + m + j; }
    __host__ __device__ int g(int j) const { return (m + 1) * m + 2 * m + j; }
    __host__ __device__ int y(int j) const { return (m + 1) * m + 3 * m + 1 + j; }
    __host__ __device__ int size() const { return (m + 1) * m + 4 * m + 1; }
};
// cycle start: beta_c = ||r_c||; a case is active if c < ncase and
// beta_c > ttol_c.  out[0..KB) = beta, out[KB] = active count.
__global__ void k_gm_start_blk(GmL L, int KB, int ncase, double* __restrict__ st, const double* __restrict__ beta,
                               const double* __restrict__ ttol, int* __restrict__ act, int* __restrict__ kd,
                               double* __restrict__ out) {
    __shared__ int cnt;
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    const int c = threadIdx.x;
    if (c < KB) {
        double* s = st + (long)c * L.size();
        const double b = beta[c];
        for (int j = 0; j <= L.m; j++) s[L.g(j)] = 0.0;
        s[L.g(0)] = b;
        const int a = (c < ncase && b > ttol[c]) ? 1 : 0;
        act[c] = a;
        kd[c] = 0;
        out[c] = b;
        if (a) atomicAdd(&cnt, 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) out[KB] = cnt;
}
// column j for every active case: hcol[i*KB + c] (i <= j+1, entry j+1 =
// ||w_c||); rotate, new Givens rotation, residual estimate; a case whose
// estimate drops to ttol (or whose Krylov space is exhausted) stops with
// kd = j+1.  out[0] = cases still active, out[1] = largest estimate.
__global__ void k_gm_givens_blk(GmL L, int KB, int j, const double* __restrict__ hcol, double* __restrict__ st,
                                const double* __restrict__ ttol, int* __restrict__ act, int* __restrict__ kd,
                                double* __restrict__ out) {
    __shared__ int cnt;
    __shared__ double rmax;
    if (threadIdx.x == 0) { cnt = 0; rmax = 0.0; }
    __syncthreads();
    const int c = threadIdx.x;
    if (c < KB && act[c]) {
        double* s = st + (long)c * L.size();
        for (int i = 0; i <= j + 1; i++) s[L.H(i, j)] = hcol[(long)i * KB + c];
        for (int i = 0; i < j; i++) {
            const double cc = s[L.cs(i)], sn = s[L.sn(i)];
            const double t1 = s[L.H(i, j)], t2 = s[L.H(i + 1, j)];
            s[L.H(i, j)] = cc * t1 + sn * t2;
            s[L.H(i + 1, j)] = -sn * t1 + cc * t2;
        }
        const double hjj = s[L.H(j, j)], hj1 = s[L.H(j + 1, j)];
        const double den = sqrt(hjj * hjj + hj1 * hj1);
        double cc = 1.0, sn = 0.0;
        if (den != 0.0) { cc = hjj / den; sn = hj1 / den; }
        s[L.cs(j)] = cc;
        s[L.sn(j)] = sn;
        s[L.H(j, j)] = cc * hjj + sn * hj1;
        s[L.H(j + 1, j)] = 0.0;
        const double gj = s[L.g(j)];
        s[L.g(j + 1)] = -sn * gj;
        s[L.g(j)] = cc * gj;
        const double res = fabs(sn * gj);
        if (!(res > ttol[c]) || hj1 == 0.0 || !isfinite(res)) {
            act[c] = 0;
            kd[c] = j + 1;
        } else {
            atomicAdd(&cnt, 1);
        }
        // largest estimate for the host's breakdown check (a NaN propagates)
        if (!isfinite(res)) rmax = res;
        else atomicMax(reinterpret_cast<unsigned long long*>(&rmax), (unsigned long long)__double_as_longlong(res));
    }
    __syncthreads();
    if (threadIdx.x == 0) { out[0] = cnt; out[1] = rmax; }
}
// y = R^-1 g per case over kd_c columns (kd_c = kdone for cases still active)
__global__ void k_gm_solve_blk(GmL L, int KB, int kdone, double* __restrict__ st, const int* __restrict__ act,
                               int* __restrict__ kd) {
    const int c = threadIdx.x;
    if (c >= KB) return;
    const int k = act[c] ? kdone : kd[c];
    kd[c] = k;
    double* s = st + (long)c * L.size();
    for (int i = k - 1; i >= 0; i--) {
        double v = s[L.g(i)];
        for (int q = i + 1; q < k; q++) v -= s[L.H(i, q)] * s[L.y(q)];
        s[L.y(i)] = v / s[L.H(i, i)];
    }
}

// ----------------------------------------------------------------- block FGMRES (host)
constexpr int kRedBlocksB = 1184;

template <int KB>
static int mdot_blk(Ctx& c, int nv, const double* V, long ld, const double* w, double* out) {
    const long nf = (long)c.ndof * KB;
    constexpr int CH = KB >= 16 ? 8 : 16;
    for (int j0 = 0; j0 < nv; j0 += CH) {
        const int k = std::min(CH, nv - j0);
        const double* Vj = V + (size_t)j0 * ld;
        if (k <= 8) k_mdot_blk<8, KB><<<kRedBlocksB, 256, 0, c.s>>>(nf, k, Vj, ld, w, c.red.p);
        else if (k <= 16) k_mdot_blk<16, KB><<<kRedBlocksB, 256, 0, c.s>>>(nf, k, Vj, ld, w, c.red.p);
        else k_mdot_blk<CH, KB><<<kRedBlocksB, 256, 0, c.s>>>(nf, k, Vj, ld, w, c.red.p);
        note_launch();
        k_final_blk<<<1, 1024, 0, c.s>>>(kRedBlocksB, k * KB, c.red.p, out + (size_t)j0 * KB, 0), note_launch();
        TCK(cudaGetLastError());
    }
    return 0;
}
template <int KB>
static int orth_blk(Ctx& c, int nv, const double* V, long ld, const double* h, double* w, double* nrm_out) {
    const long nf = (long)c.ndof * KB;
    constexpr int CH = KB >= 16 ? 8 : 16;
    for (int j0 = 0; j0 < nv; j0 += CH) {
        const int k = std::min(CH, nv - j0);
        const double* Vj = V + (size_t)j0 * ld;
        const double* hj = h + (size_t)j0 * KB;
        if (k <= 8) k_orth_blk<8, KB><<<kRedBlocksB, 256, 0, c.s>>>(nf, k, Vj, ld, hj, w, c.red.p);
        else if (k <= 16) k_orth_blk<16, KB><<<kRedBlocksB, 256, 0, c.s>>>(nf, k, Vj, ld, hj, w, c.red.p);
        else k_orth_blk<CH, KB><<<kRedBlocksB, 256, 0, c.s>>>(nf, k, Vj, ld, hj, w, c.red.p);
        note_launch();
    }
    // the last sweep's partials hold ||w_c||^2 of the fully orthogonalised w
    k_final_blk<<<1, 32 * KB, 0, c.s>>>(kRedBlocksB, KB, c.red.p, nrm_out, 1), note_launch();
    TCK(cudaGetLastError());
    return 0;
}
// per-case norms of a block vector -> out[KB]
template <int KB>
static int norms_blk(Ctx& c, const double* w, double* out) {
    const long nf = (long)c.ndof * KB;
    k_mdot_blk<8, KB><<<kRedBlocksB, 256, 0, c.s>>>(nf, 1, w, 0, w, c.red.p), note_launch();
    k_final_blk<<<1, 32 * KB, 0, c.s>>>(kRedBlocksB, KB, c.red.p, out, 1), note_launch();
    TCK(cudaGetLastError());
    return 0;
}

// Autotuning of the block operator's CTAs per SM (1 or the occupancy
// limit), timed on this context's operator at its first block solve.
// the level-0 block sweep's slot-group form (1 or 3 slots per load group),
// timed on the context's own operator (MODE 0 on scratch rows of the basis)
template <class T, int KB>
static int tune_sell_u(Ctx& c, cudaEvent_t e0, cudaEvent_t e1) {
    if (!avals<T>(c).A0s.p) return 0;
    const long nf = (long)c.ndof * KB;
    const T* x = reinterpret_cast<const T*>(c.blk.V.p);
    T* y = reinterpret_cast<T*>(c.blk.V.p + nf);
    double best = 1e30;
    int pick = 1;
    for (int u : {1, 3}) {
        c.tune.blk_sell_u = u;
        double t = 1e30;
        for (int rep = 0; rep < 3; rep++) {
            TCK(cudaEventRecord(e0, c.s));
            launch_sell_blk<T, KB, 0>(c, x, y, nullptr, nullptr, nullptr, nullptr, nullptr, 0, 0);
            TCK(cudaEventRecord(e1, c.s));
            TCK(cudaEventSynchronize(e1));
            float ms = 0.f;
            TCK(cudaEventElapsedTime(&ms, e0, e1));
            t = std::min(t, (double)ms);
        }
        if (t < best) { best = t; pick = u; }
    }
    c.tune.blk_sell_u = pick;
    return 0;
}
template <class T>
static int tune_sell_u_kb(Ctx& c, cudaEvent_t e0, cudaEvent_t e1) {
    if (c.blk.kb == 4) return tune_sell_u<T, 4>(c, e0, e1);
    if (c.blk.kb == 8) return tune_sell_u<T, 8>(c, e0, e1);
    return tune_sell_u<T, 16>(c, e0, e1);
}

int autotune_block(Ctx& c) {
    BlockState& B = c.blk;
    if (!tuning_on(c) || c.tune.block_done || !B.V.p) return 0;
    c.tune.block_done = true;
    const long nf = (long)c.ndof * B.kb;
    double* u = B.V.p;
    double* y = B.V.p + nf;
    TCK(cudaMemsetAsync(u, 0, sizeof(double) * 2 * nf, c.s));
    const bool prof = c.prof.on;
    c.prof.on = false;
    cudaEvent_t e0, e1;
    TCK(cudaEventCreate(&e0));
    TCK(cudaEventCreate(&e1));
    double best = 1e30;
    int pick = 0, pick_st = 3;
    for (int cand : {31, 30, 21, 20}) {  // Ke copies in flight per warp x 10 + CTAs per SM (0: occupancy)
        if (c.p.blk_stages && cand / 10 != c.p.blk_stages) continue;  // forced by the options
        const int ctas = cand % 10;
        c.tune.blk_ctas = ctas;
        c.tune.blk_stages = cand / 10;
        double t = 1e30;
        for (int rep = 0; rep < 3; rep++) {
            TCK(cudaEventRecord(e0, c.s));
            TRET(blk_apply(c, u, y, nullptr, 1.0));
            TCK(cudaEventRecord(e1, c.s));
            TCK(cudaEventSynchronize(e1));
            float ms = 0.f;
            TCK(cudaEventElapsedTime(&ms, e0, e1));
            t = std::min(t, (double)ms);
        }
        if (t < best) { best = t; pick = ctas; pick_st = cand / 10; }
    }
    const int rc = c.p.precision == TOPO_PREC_MIXED ? tune_sell_u_kb<float>(c, e0, e1) : tune_sell_u_kb<double>(c, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    TRET(rc);
    c.tune.blk_ctas = pick;
    c.tune.blk_stages = pick_st;
    c.prof.on = prof;
    c.info.tuned[3] = 10 * pick_st + pick;
    return 0;
}

// Arnoldi step j for all cases (see the single-load step in solver.cu)
struct BlkStepArgs {
    int j;
    long nf;
    GmL GL;
    double *hcol, *st, *ttol_d, *out, *hs;
    int *act, *kd;
};
template <int KB>
static int arnoldi_step_blk(Ctx& c, void* p) {
    const BlkStepArgs& a = *static_cast<const BlkStepArgs*>(p);
    BlockState& B = c.blk;
    const int j = a.j;
    const long nf = a.nf;
    const double* vj = B.V.p + (size_t)j * nf;
    TRET(precond_blk(c, vj, j));
    if (c.p.precision == TOPO_PREC_MIXED) TRET(blk_apply_f32in(c, B.Z32.p + (size_t)j * nf, B.w.p, nullptr, 1.0));
    else TRET(blk_apply(c, B.Z64.p + (size_t)j * nf, B.w.p, nullptr, 1.0));
    TRET(mdot_blk<KB>(c, j + 1, B.V.p, nf, B.w.p, a.hcol));
    TRET(orth_blk<KB>(c, j + 1, B.V.p, nf, a.hcol, B.w.p, a.hcol + (size_t)(j + 1) * KB));
    k_scale_blk<KB><<<grid_for(nf, 256), 256, 0, c.s>>>(nf, B.w.p, a.hcol + (size_t)(j + 1) * KB, a.act,
                                                      B.V.p + (size_t)(j + 1) * nf), note_launch();
    k_gm_givens_blk<<<1, 32, 0, c.s>>>(a.GL, KB, j, a.hcol, a.st, a.ttol_d, a.act, a.kd, a.out + 2 * j), note_launch();
    TCK(cudaMemcpyAsync(a.hs + 2 * j, a.out + 2 * j, 2 * sizeof(double), cudaMemcpyDeviceToHost, c.s));
    TCK(cudaGetLastError());
    return 0;
}

template <int KB>
static int fgmres_blk(Ctx& c, const double* b, double* x, int* its_out, int* status) {
    BlockState& B = c.blk;
    const long nf = (long)c.ndof * KB;
    const int m = std::max(1, std::min(c.p.fem_restart, 128));
    const int maxit = c.p.fem_maxit;
    const GmL GL{m};
    const bool mixed = c.p.precision == TOPO_PREC_MIXED;
    if (!B.V.p || B.V.n < (size_t)(m + 1) * nf) {
        TRET(B.V.alloc((size_t)(m + 1) * nf));
        TRET(B.w.alloc(nf));
        B.Z32.reset();
        B.Z64.reset();
    }
    if (mixed && !B.Z32.p) TRET(B.Z32.alloc((size_t)m * nf));
    if (!mixed && !B.Z64.p) TRET(B.Z64.alloc((size_t)m * nf));
    const size_t ssz = (size_t)KB * GL.size();
    if (B.st.n < ssz + 8 * (size_t)(m + 2) * KB + 64) TRET(B.st.alloc(ssz + 8 * (size_t)(m + 2) * KB + 64));
    if (B.ik.n < (size_t)4 * KB) TRET(B.ik.alloc(4 * KB));
    if ((long)c.red.n < kRedBlocksB * 32L * KB) TRET(c.red.alloc(kRedBlocksB * 32L * KB));
    while ((int)c.gm_ev.size() < m + 1) {
        cudaEvent_t e;
        TCK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        c.gm_ev.push_back(e);
    }
    if (!B.hs.h || B.hs.n < (size_t)(4 * (m + 2) + 4 * KB + 40)) TRET(B.hs.alloc(4 * (m + 2) + 4 * KB + 40));
    double* st = B.st.p;                       // KB Arnoldi states
    double* hcol = st + ssz;                   // (m+2) x KB Hessenberg column
    double* ttol_d = hcol + (size_t)(m + 2) * KB;
    double* beta_d = ttol_d + KB;
    double* out = beta_d + KB;                 // per-iteration outputs (2 each), then start outputs
    double* out_start = out + 2 * (m + 1);
    int* act = B.ik.p;
    int* kd = B.ik.p + KB;
    double* hs = B.hs.h;
    TRET(blk_setup(c));
    TRET(autotune_block(c));
    // the V-cycle work vectors and the slot moduli exist before any capture
    // (a captured step must not depend on host-side state that changes)
    if (mixed) TRET(alloc_bvecs<float>(c));
    else TRET(alloc_bvecs<double>(c));
    TRET(blk_setup(c));
    // buffers and options the Arnoldi-step graphs depend on
    uint64_t sig = 0x2b1c0ffeeull;
    for (uint64_t v : {(uint64_t)(uintptr_t)B.V.p, (uint64_t)(uintptr_t)B.Z32.p, (uint64_t)(uintptr_t)B.Z64.p,
                       (uint64_t)(uintptr_t)B.w.p, (uint64_t)(uintptr_t)B.st.p, (uint64_t)(uintptr_t)B.ik.p,
                       (uint64_t)(uintptr_t)B.hs.h, (uint64_t)(uintptr_t)c.red.p, (uint64_t)(uintptr_t)B.Es.p,
                       (uint64_t)(uintptr_t)B.bv32.x[0].p, (uint64_t)(uintptr_t)B.bv64.x[0].p,
                       (uint64_t)(uintptr_t)c.v32.A0s.p, (uint64_t)(uintptr_t)c.v64.A0s.p,
                       (uint64_t)(uintptr_t)c.cinv.p, (uint64_t)(uintptr_t)c.rho.p, (uint64_t)c.p.precision,
                       (uint64_t)m, (uint64_t)c.nlev, (uint64_t)c.p.cheb_degree, (uint64_t)c.p.cheb_degree_post, (uint64_t)c.p.cheb_degree_coarse, (uint64_t)c.tune.blk_ctas, (uint64_t)c.tune.blk_stages, (uint64_t)c.tune.blk_sell_u, (uint64_t)KB, (uint64_t)nf})
        sig = sig_mix(sig, v);
    StepGraphs& G = B.graphs;
    if (G.sig != sig) {
        G.drop();
        G.sig = sig;
    }
    const bool capture_ok = c.p.fem_graphs && G.seen == sig;
    G.seen = sig;
    // ||b_c|| -> stopping thresholds max(rtol ||b_c||, 1e-50)
    TRET(norms_blk<KB>(c, b, beta_d));
    TCK(cudaMemcpyAsync(hs, beta_d, KB * sizeof(double), cudaMemcpyDeviceToHost, c.s));
    TCK(cudaStreamSynchronize(c.s));
    double ttol[16];
    for (int k = 0; k < KB; k++) ttol[k] = std::max(c.p.fem_rtol * hs[k], 1e-50);
    TCK(cudaMemcpyAsync(ttol_d, ttol, KB * sizeof(double), cudaMemcpyHostToDevice, c.s));
    TCK(cudaStreamSynchronize(c.s));
    int its = 0;
    bool conv = false;
    while (!conv && its < maxit) {
        // r = b - K x, beta_c = ||r_c||
        TRET(blk_apply(c, x, B.w.p, b, -1.0));
        TRET(norms_blk<KB>(c, B.w.p, beta_d));
        k_gm_start_blk<<<1, 32, 0, c.s>>>(GL, KB, c.ncases, st, beta_d, ttol_d, act, kd, out_start), note_launch();
        TCK(cudaMemcpyAsync(hs + 2 * (m + 2), out_start, (KB + 1) * sizeof(double), cudaMemcpyDeviceToHost, c.s));
        TCK(cudaStreamSynchronize(c.s));
        for (int k = 0; k < c.ncases; k++)
            if (!std::isfinite(hs[2 * (m + 2) + k])) { set_error("block FGMRES residual is not finite"); return TOPO_ERR_NAN; }
        if (hs[2 * (m + 2) + KB] == 0.0) { conv = true; break; }
        k_scale_blk<KB><<<grid_for(nf, 256), 256, 0, c.s>>>(nf, B.w.p, beta_d, act, B.V.p), note_launch();
        const int jmax = std::min(m, maxit - its);
        int kdone = jmax;
        bool stop = false;
        for (int j = 0; j <= jmax && !stop; j++) {
            if (j < jmax) {
                BlkStepArgs sa{j, nf, GL, hcol, st, ttol_d, out, hs, act, kd};
                TRET(step_graph_run(c, G, j, capture_ok, arnoldi_step_blk<KB>, &sa));
                TCK(cudaEventRecord(c.gm_ev[j], c.s));
            }
            if (j == 0) continue;
            // check iteration j-1 while iteration j runs
            TCK(cudaEventSynchronize(c.gm_ev[j - 1]));
            its++;
            const double nact = hs[2 * (j - 1)], rmax = hs[2 * (j - 1) + 1];
            if (!std::isfinite(rmax)) { set_error("block FGMRES breakdown (non-finite residual)"); return TOPO_ERR_NAN; }
            if (nact == 0.0) {
                kdone = j;
                stop = true;
                conv = true;
            }
        }
        k_gm_solve_blk<<<1, 32, 0, c.s>>>(GL, KB, kdone, st, act, kd), note_launch();
        if (mixed)
            k_update_blk<float, KB><<<grid_for(nf, 256), 256, 0, c.s>>>(nf, B.Z32.p, nf, st, GL.size(), GL.y(0), kd, x),
                note_launch();
        else
            k_update_blk<double, KB><<<grid_for(nf, 256), 256, 0, c.s>>>(nf, B.Z64.p, nf, st, GL.size(), GL.y(0), kd,
                                                                         x), note_launch();
        TCK(cudaGetLastError());
    }
    TRET(blk_check_error(c));
    *its_out = its;
    *status = conv ? 0 : 1;
    return 0;
}

template <int KB>
static int true_residuals(Ctx& c, double* nr) {
    BlockState& B = c.blk;
    TRET(blk_apply(c, B.U.p, B.w.p, B.F.p, -1.0));
    TRET(norms_blk<KB>(c, B.w.p, nr));
    return norms_blk<KB>(c, B.F.p, nr + 16);
}

// K(x) [u_1..u_k] = [f_1..f_k] for all load cases at once; u ([case][ndof])
// receives the solutions, the block copy stays in blk.U for the
// sensitivities.
int fem_solve_block(Ctx& c, const double* xphys, double* u) {
    TRET(compute_moduli(c, xphys));
    TRET(amg_numeric(c));
    TRET(blk_setup(c));
    BlockState& B = c.blk;
    const int KB = B.kb;
    const long nf = (long)c.ndof * KB;
    if (!B.F.p) {
        TRET(B.F.alloc(nf));
        TRET(blk_interleave(c, c.F.p, B.F.p));
    }
    if (!B.U.p) TRET(B.U.alloc(nf));
    // AssembleFem zeroes U (SolveFem.cpp:333); the optional warm start keeps
    // the previous block solution
    if (!(c.p.fem_warm_start && c.u_valid && B.u_valid)) TCK(cudaMemsetAsync(B.U.p, 0, sizeof(double) * nf, c.s));
    int its = 0, st = 0;
    if (KB == 4) TRET(fgmres_blk<4>(c, B.F.p, B.U.p, &its, &st));
    else if (KB == 8) TRET(fgmres_blk<8>(c, B.F.p, B.U.p, &its, &st));
    else TRET(fgmres_blk<16>(c, B.F.p, B.U.p, &its, &st));
    B.u_valid = B.u_fresh = true;
    TRET(blk_deinterleave(c, B.U.p, u));
    // true residuals ||F_c - K U_c|| / ||F_c||, worst case reported
    double* nr = B.st.p;  // scratch (after the solve)
    if (KB == 4) TRET(true_residuals<4>(c, nr));
    else if (KB == 8) TRET(true_residuals<8>(c, nr));
    else TRET(true_residuals<16>(c, nr));
    TCK(cudaMemcpyAsync(B.hs.h, nr, 32 * sizeof(double), cudaMemcpyDeviceToHost, c.s));
    TCK(cudaStreamSynchronize(c.s));
    double rel_worst = 0.0;
    for (int k = 0; k < c.ncases; k++) {
        const double fn = B.hs.h[16 + k], rn = B.hs.h[k];
        rel_worst = std::max(rel_worst, fn > 0 ? rn / fn : rn);
    }
    if (c.p.verbose) printf("Norm of error %e, Iterations %d (%d load cases, block)\n", rel_worst, its, c.ncases);
    c.u_valid = (u == c.U.p);
    c.info.fem_its = its;
    c.info.fem_relres = rel_worst;
    c.info.fem_status = st;
    return st ? TOPO_NOT_CONVERGED : 0;
}

}  // namespace topo
