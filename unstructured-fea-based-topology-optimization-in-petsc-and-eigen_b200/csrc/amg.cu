// amg.cu -- numeric phase of the smoothed-aggregation AMG (rebuilt every
// design iteration on the device) and its V-cycle.
//
// Replaces PCGAMG with PCGAMGSetNlevels(pc,4) + PCSetCoordinates
// (SolveFem.cpp:130-132).  Per design iteration:
//   A0  <- sum_e E_e Ke_e gathered node-row by node-row (deterministic),
//          Dirichlet rows/columns identity (MatZeroRowsColumns, SolveFem.cpp:324)
//   rho <- power iteration on D^-1 A (warm-started across design iterations)
//   P   <- (I - 4/(3 rho) D^-1 A) Pt        (smoothed aggregation)
//   A+  <- P^T (A P)                         (Galerkin, two fixed-pattern SpGEMMs
//                                             from host-built per-mesh pair plans)
//   coarsest: explicit FP64 inverse (Gauss-Jordan, partial pivoting)
// V-cycle: Chebyshev(k)-Jacobi pre/post smoothing on [0.1, 1.1] rho; level 0
// on a sliced-ELLPACK copy of A0 whose sweeps fetch the next slot group's
// column ids while gathering the current group; levels >= 1 on BSR with a
// tuned number of lanes per block row; prolongation with one packed P block
// per lane; every V-cycle kernel started early by programmatic dependent
// launch (it waits on the GPU for its predecessor's output).
//
// BSR values are slot-interleaved (see ctx.h) so that the lanes of a warp
// walking the blocks of one row read every block entry as a coalesced run.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>

#include "ctx.h"

namespace topo {

int kmatvec32(Ctx& c, const float* u, float* y, const float* b);
int kmatvec64r(Ctx& c, const double* u, double* y, const double* b);

__host__ __device__ __forceinline__ int pk_index_amg(int i, int j, int n) {
    if (i > j) { int t = i; i = j; j = t; }
    return i * n - (i * (i - 1)) / 2 + (j - i);
}

// ----------------------------------------------------------------- level-0 assembly
// Node-row copy of the element matrices, built once per mesh: for n2e
// position p (n2e[p] = e * NEN + l) the three rows of local node l of Ke(e),
// 3 x 3NEN values in one contiguous run, so the assembly below reads each
// (node, element) pair with coalesced loads instead of one scattered
// 4-byte load per 128-byte line of the element-major (AoSoA) matrices.
template <class T, int NEN>
__global__ void k_ke_node_rows(long np, const int* __restrict__ n2e, const T* __restrict__ ke, T* __restrict__ kst) {
    constexpr int ND = 3 * NEN, NPK = ND * (ND + 1) / 2, W = 3 * ND;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < np * W; t += (long)gridDim.x * blockDim.x) {
        const long p = t / W;
        const int r = (int)(t - p * W), cc = r / ND, k = r % ND;
        const int q = n2e[p], e = q / NEN, l = q % NEN;
        kst[t] = ke[((size_t)(e >> 5) * NPK + pk_index_amg(cc * NEN + l, k, ND)) * 32 + (e & 31)];
    }
}

// One warp per node row: lane k owns column k of the element's 3*NEN columns
// and adds the node's three rows into a shared-memory row buffer, element by
// element in n2e order (so the sum order is fixed); the loads of four
// elements are issued together before their sums.  The row is then written
// out with the Dirichlet identity applied.
template <class T, int NEN>
__global__ void k_assemble_A0(int nn, const int* __restrict__ n2e_ptr, const int* __restrict__ n2e,
                              const uint16_t* __restrict__ bpos, const T* __restrict__ kst, const T* __restrict__ Ee,
                              const int* __restrict__ rp, const int* __restrict__ ci,
                              const unsigned char* __restrict__ dfix, T* __restrict__ A, int maxdeg,
                              T* __restrict__ S, const int* __restrict__ sp) {
    constexpr int ND = 3 * NEN, U = 4;
    static_assert(ND <= 32, "one lane per element column");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.x * (blockDim.x >> 5) + wib;
    if (i >= nn) return;
    T* buf = reinterpret_cast<T*>(smem_raw) + (size_t)wib * maxdeg * 9;
    const int r0 = rp[i], nb = rp[i + 1] - r0;
    for (int q = lane; q < 9 * nb; q += 32) buf[q] = T(0);
    __syncwarp();
    const int m = lane % NEN, d = lane / NEN;
    const int pbeg = n2e_ptr[i], pend = n2e_ptr[i + 1];
    for (int pc = pbeg; pc < pend; pc += 32) {
        const int np = min(32, pend - pc);
        const int myq = lane < np ? n2e[pc + lane] : 0;  // (element, local node) of the chunk, one per lane
        for (int u0 = 0; u0 < np; u0 += U) {
            T val[U][3], Eu[U];
            int slot[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int q = __shfl_sync(0xffffffffu, myq, (u0 + u) & 31);
                slot[u] = 0;
                Eu[u] = val[u][0] = val[u][1] = val[u][2] = T(0);
                if (u0 + u < np && lane < ND) {
                    const int e = q / NEN, l = q % NEN;
                    Eu[u] = Ee[e];
                    const T* kr = kst + (size_t)(pc + u0 + u) * 3 * ND;
                    slot[u] = bpos[((size_t)e * NEN + l) * NEN + m];
#pragma unroll
                    for (int cc = 0; cc < 3; cc++) val[u][cc] = kr[cc * ND + lane];
                }
            }
            // two lanes may add into the same row entry for different
            // elements: each element's adds are separated by a warp barrier
#pragma unroll
            for (int u = 0; u < U; u++) {
                if (u0 + u < np && lane < ND)
#pragma unroll
                    for (int cc = 0; cc < 3; cc++) buf[(cc * 3 + d) * nb + slot[u]] += Eu[u] * val[u][cc];
                __syncwarp();
            }
        }
    }
    __syncwarp();
    for (int idx = lane; idx < 9 * nb; idx += 32) {
        const int ent = idx / nb, slot = idx - ent * nb;
        const int cc = ent / 3, dd = ent % 3;
        const int j = ci[r0 + slot];
        T v = buf[idx];
        const bool rf = dfix[3L * i + cc], cf = dfix[3L * j + dd];
        if (rf || cf) v = (rf && j == i && cc == dd) ? T(1) : T(0);
        A[(size_t)r0 * 9 + idx] = v;
        // the smoother's sliced-ELLPACK copy (its padding stays zero)
        if (S) S[sell_idx<T>((size_t)(sp[i >> 5] >> 5) + slot, ent, i & 31)] = v;
    }
}

// dinv[dof] = 1 / A_dof,dof (point Jacobi)
template <class T, int BS>
__global__ void k_diag_inv(int nnode, const int* __restrict__ rp, const int* __restrict__ diagpos,
                           const T* __restrict__ A, T* __restrict__ dinv) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nnode) return;
    const int r0 = rp[i], nb = rp[i + 1] - r0, s = diagpos[i];
#pragma unroll
    for (int cc = 0; cc < BS; cc++) {
        T a = A[(size_t)r0 * BS * BS + (cc * BS + cc) * nb + s];
        dinv[(long)BS * i + cc] = a != T(0) ? T(1) / a : T(1);
    }
}

// ----------------------------------------------------------------- BSR SpMV
// G lanes per block row.  mode 0: y = A x; 1: y = b - A x; 2: y += A x;
// 3 (power iteration): y = sigma * Dinv A x with sigma = *scal;
// 5 (restriction into a level that is smoothed next): y = A x, and the
// level's first Chebyshev step from a zero guess on the same rows (the
// operations of k_cheb_first): r5 = y, d5 = x5 = Dinv y / (0.6 *scal).
template <class T, int BR, int BC, int G>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 2) k_bsr_spmv(int nrows, const int* __restrict__ rp, const int* __restrict__ ci, const T* __restrict__ A,
                           const T* __restrict__ x, T* __restrict__ y, const T* __restrict__ b, int mode,
                           const T* __restrict__ dinv, const double* __restrict__ scal, T* __restrict__ r5,
                           T* __restrict__ d5, T* __restrict__ x5) {
    pdl_trigger();
    const int gid = (blockIdx.x * blockDim.x + threadIdx.x) / G;
    const int gl = threadIdx.x % G;
    const bool active = gid < nrows;
    const long o = (long)BR * gid + gl;
    int r0 = 0, nb = 0;
    if (active) {
        r0 = rp[gid];
        nb = rp[gid + 1] - r0;
    }
    pdl_wait();
    // the epilogue's own operand, loaded ahead of the row's products
    T pre = T(0);
    if (active && gl < BR) {
        if (mode == 1) pre = b[o];
        else if (mode == 2) pre = y[o];
        else if (mode >= 3) pre = dinv[o];
    }
    T acc[BR];
#pragma unroll
    for (int r = 0; r < BR; r++) acc[r] = T(0);
    if (active) {
        const T* Ar = A + (size_t)r0 * BR * BC;
        // the next block's column id is fetched while this block is summed:
        // one memory round trip per block instead of two
        int j = gl < nb ? ci[r0 + gl] : 0;
        for (int s = gl; s < nb; s += G) {
            const int jn = s + G < nb ? ci[r0 + s + G] : 0;
            T xv[BC];
#pragma unroll
            for (int d = 0; d < BC; d++) xv[d] = x[(long)BC * j + d];
#pragma unroll
            for (int r = 0; r < BR; r++)
#pragma unroll
                for (int d = 0; d < BC; d++) acc[r] += Ar[(r * BC + d) * nb + s] * xv[d];
            j = jn;
        }
    }
#pragma unroll
    for (int r = 0; r < BR; r++)
#pragma unroll
        for (int off = G / 2; off > 0; off >>= 1) acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], off);
    if (active && gl < BR) {
        T v = T(0);
#pragma unroll
        for (int r = 0; r < BR; r++)
            if (r == gl) v = acc[r];
        if (mode == 0) y[o] = v;
        else if (mode == 1) y[o] = pre - v;
        else if (mode == 2) y[o] = pre + v;
        else if (mode == 4) y[o] += pre * v;  // row-scaled prolongation into hat variables
        else if (mode == 5) {
            y[o] = v;
            r5[o] = v;
            const T it = T(1.0 / (0.6 * (*scal)));
            const T di = pre * v * it;
            d5[o] = di;
            x5[o] = di;
        } else y[o] = T(*scal) * pre * v;
    }
}

// ----------------------------------------------------------------- prolongation, one block per lane
// Packed block-major layout: entry e of block g sits in 16-byte group e / VPL
// (VPL = 16 / sizeof(T) entries per group), groups of all blocks stored one
// after another, so lane g of a warp reads its block's group as one 16-byte
// load and the warp's loads are contiguous; a remainder of fewer than VPL
// entries (FP32 3x6 blocks: 2) forms one more, narrower group.
template <class T, int BB>
__host__ __device__ __forceinline__ size_t pk_off(int e, long g, long npad) {
    constexpr int VPL = 16 / (int)sizeof(T), NG = BB / VPL, REM = BB - NG * VPL;
    if (e < NG * VPL) return (size_t)(e / VPL) * npad * VPL + (size_t)g * VPL + (e % VPL);
    return (size_t)NG * npad * VPL + (size_t)g * REM + (e - NG * VPL);
}

template <class T, int BB>
__global__ void k_bsr_pack(int nrows, const int* __restrict__ rp, const T* __restrict__ A, T* __restrict__ Pk,
                           long npad) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (i >= nrows) return;
    const int r0 = rp[i], nb = rp[i + 1] - r0;
    for (int q = lane; q < BB * nb; q += 32) {
        const int e = q / nb, s = q - e * nb;
        Pk[pk_off<T, BB>(e, (long)r0 + s, npad)] = A[(size_t)r0 * BB + q];
    }
}

// y += P x (mode 2) or y += dinv (P x) (mode 4, hat variables) with P packed:
// warp w owns rows [wrow[w], wrow[w+1]) -- at most 32 rows whose blocks
// (at most 32) are blocks rp[wrow[w]] .. of the packed array -- one block per
// lane.  Each lane finds its row by a binary search over the row starts held
// one per lane, and a segmented shuffle reduction leaves each row's sum in
// the row's first lane.  Rows without blocks are skipped (nothing to add).
template <class T, int BR, int BC>
__global__ void __launch_bounds__(256) k_bsr_lane(int nw, const int* __restrict__ wrow, const int* __restrict__ rp,
                                                  const int* __restrict__ ci, const T* __restrict__ Pk, long npad,
                                                  const T* __restrict__ x, T* __restrict__ y, int mode,
                                                  const T* __restrict__ dinv) {
    constexpr int BB = BR * BC, VPL = 16 / (int)sizeof(T), NG = BB / VPL, REM = BB - NG * VPL;
    static_assert(BC % 2 == 0, "column blocks are read as pairs");
    pdl_trigger();
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= nw) return;  // uniform per warp
    const int ra = wrow[w], nr = wrow[w + 1] - ra;
    const int g0 = rp[ra], nblk = rp[ra + nr] - g0;
    const int my_start = lane < nr ? rp[ra + lane] - g0 : 64;  // start lane of row ra + lane
    // row of this lane's block: last row whose start <= lane (an empty row
    // shares its start with the next row, which the search then picks)
    int lo = 0, hi = nr - 1;
#pragma unroll
    for (int it = 0; it < 5; it++) {
        const int mid = (lo + hi + 1) >> 1;
        const int sm = __shfl_sync(0xffffffffu, my_start, mid);
        if (lo < hi) {
            if (sm <= lane) lo = mid;
            else hi = mid - 1;
        }
    }
    const int row = lo;
    const int seg_start = __shfl_sync(0xffffffffu, my_start, row);
    const int nxt = __shfl_sync(0xffffffffu, my_start, row + 1 < 32 ? row + 1 : 31);
    const int seg_end = row + 1 < nr ? nxt : nblk;
    T acc[BR];
#pragma unroll
    for (int r = 0; r < BR; r++) acc[r] = T(0);
    // pattern and values are fixed during the solve: fetched before the wait
    const long g = (long)g0 + lane;
    int j = 0;
    T v[BB];
    if (lane < nblk) {
        j = __ldg(ci + g);
#pragma unroll
        for (int k = 0; k < NG; k++) {
            const uint4 t = __ldg(reinterpret_cast<const uint4*>(Pk + (size_t)k * npad * VPL + (size_t)g * VPL));
            memcpy(v + k * VPL, &t, 16);
        }
#pragma unroll
        for (int k = 0; k < REM; k++) v[NG * VPL + k] = Pk[(size_t)NG * npad * VPL + (size_t)g * REM + k];
    }
    pdl_wait();
    if (lane < nblk) {
        T xv[BC];
#pragma unroll
        for (int d = 0; d < BC; d += 2) {
            if constexpr (sizeof(T) == 4) {
                const float2 t = __ldg(reinterpret_cast<const float2*>(x + (long)BC * j + d));
                xv[d] = t.x;
                xv[d + 1] = t.y;
            } else {
                const double2 t = __ldg(reinterpret_cast<const double2*>(x + (long)BC * j + d));
                xv[d] = t.x;
                xv[d + 1] = t.y;
            }
        }
#pragma unroll
        for (int r = 0; r < BR; r++)
#pragma unroll
            for (int d = 0; d < BC; d++) acc[r] += v[r * BC + d] * xv[d];
    }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1)
#pragma unroll
        for (int r = 0; r < BR; r++) {
            const T t = __shfl_down_sync(0xffffffffu, acc[r], o);
            if (lane + o < seg_end) acc[r] += t;
        }
    if (lane < nblk && lane == seg_start) {
        const long o = (long)BR * (ra + row);
#pragma unroll
        for (int r = 0; r < BR; r++) {
            if (mode == 2) y[o + r] += acc[r];
            else y[o + r] += dinv[o + r] * acc[r];
        }
    }
}

// fused Chebyshev step on a BSR level: t = A dold; r -= t;
// dnew = c1 dold + c2 Dinv r; x += dnew (c1, c2 from rho and the step's
// recurrence numbers cr = rho_k rho_{k-1}, cq = 2 rho_k)
template <class T, int BS, int G>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? (BS <= 3 ? 5 : 4) : 2) k_bsr_cheb(int nrows, const int* __restrict__ rp, const int* __restrict__ ci, const T* __restrict__ A,
                           const T* __restrict__ dold, T* __restrict__ dnew, T* __restrict__ r, T* __restrict__ x,
                           const T* __restrict__ dinv, const double* __restrict__ rho, double cr, double cq) {
    pdl_trigger();
    const int gid = (blockIdx.x * blockDim.x + threadIdx.x) / G;
    const int gl = threadIdx.x % G;
    const bool active = gid < nrows;
    const long o = (long)BS * gid + gl;
    int r0 = 0, nb = 0;
    T r_o = T(0), d_o = T(0), di_o = T(0);
    if (active) {
        r0 = rp[gid];
        nb = rp[gid + 1] - r0;
        if (gl < BS) di_o = dinv[o];
    }
    pdl_wait();
    // the update's own operands, loaded ahead of the row's products
    if (active && gl < BS) {
        r_o = r[o];
        d_o = dold[o];
    }
    T acc[BS];
#pragma unroll
    for (int q = 0; q < BS; q++) acc[q] = T(0);
    if (active) {
        const T* Ar = A + (size_t)r0 * BS * BS;
        int j = gl < nb ? ci[r0 + gl] : 0;  // next column id prefetched as in k_bsr_spmv
        for (int s = gl; s < nb; s += G) {
            const int jn = s + G < nb ? ci[r0 + s + G] : 0;
            T xv[BS];
#pragma unroll
            for (int d = 0; d < BS; d++) xv[d] = dold[(long)BS * j + d];
#pragma unroll
            for (int q = 0; q < BS; q++)
#pragma unroll
                for (int d = 0; d < BS; d++) acc[q] += Ar[(q * BS + d) * nb + s] * xv[d];
            j = jn;
        }
    }
#pragma unroll
    for (int q = 0; q < BS; q++)
#pragma unroll
        for (int off = G / 2; off > 0; off >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], off);
    if (active && gl < BS) {
        T v = T(0);
#pragma unroll
        for (int q = 0; q < BS; q++)
            if (q == gl) v = acc[q];
        const double delta = 0.5 * (*rho);
        const T c2 = T(cq / delta);
        T rn = r_o - v;
        T dn = T(cr) * d_o + c2 * di_o * rn;
        r[o] = rn;
        dnew[o] = dn;
        x[o] += dn;
    }
}

// ----------------------------------------------------------------- level-0 sliced ELLPACK
// One thread per node row; block k of the rows of slice s is entry
// sp[s] + 32k + lane (column ids: one contiguous line per warp), its 9
// values in slot sp[s]/32 + k of the value array (sell_idx: two 16-byte
// vectors and one scalar per row, each a coalesced run over the warp).
// mode 0: y = A x; 1: y = b - A x; 3: y = sigma Dinv A x
// One row's product with the sliced-ELLPACK operator: w slots, U at a time,
// with the column ids of the next U slots loaded while the current U are
// gathered, so each group waits for one memory round trip (the values and
// x) instead of two (column id, then x).  BATCH issues all of a group's
// loads before its arithmetic (more bytes in flight, more registers);
// otherwise slot by slot (fewer registers, more warps per SM).
template <class T, int U, bool BATCH>
__device__ __forceinline__ void sell_row_product(const T* __restrict__ S, size_t sb, int lane, const int* __restrict__ cp,
                                                 int w, const T* __restrict__ x, T (&acc)[3]) {
    int jn[U];
#pragma unroll
    for (int u = 0; u < U; u++) jn[u] = u < w ? __ldg(cp + 32 * u) : 0;
    pdl_wait();  // x may come from the previous kernel
    for (int k = 0; k < w; k += U) {
        int jc[U];
#pragma unroll
        for (int u = 0; u < U; u++) jc[u] = jn[u];
#pragma unroll
        for (int u = 0; u < U; u++) jn[u] = k + U + u < w ? __ldg(cp + 32 * (k + U + u)) : 0;
        if constexpr (!BATCH) {
#pragma unroll
            for (int u = 0; u < U; u++) {
                if (k + u < w) {
                    const int j = jc[u];
                    const T x0 = x[3L * j], x1 = x[3L * j + 1], x2 = x[3L * j + 2];
                    T a[9];
                    sell_load9<T>(S, sb + k + u, lane, a);
                    acc[0] += a[0] * x0 + a[1] * x1 + a[2] * x2;
                    acc[1] += a[3] * x0 + a[4] * x1 + a[5] * x2;
                    acc[2] += a[6] * x0 + a[7] * x1 + a[8] * x2;
                }
            }
        } else {
            // all of the group's loads first, then its arithmetic
            T xv[U][3], av[U][9];
#pragma unroll
            for (int u = 0; u < U; u++) {
                if (k + u < w) {
                    const int j = jc[u];
                    xv[u][0] = x[3L * j];
                    xv[u][1] = x[3L * j + 1];
                    xv[u][2] = x[3L * j + 2];
                    sell_load9<T>(S, sb + k + u, lane, av[u]);
                } else {
#pragma unroll
                    for (int q = 0; q < 3; q++) xv[u][q] = T(0);
#pragma unroll
                    for (int q = 0; q < 9; q++) av[u][q] = T(0);
                }
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                acc[0] += av[u][0] * xv[u][0] + av[u][1] * xv[u][1] + av[u][2] * xv[u][2];
                acc[1] += av[u][3] * xv[u][0] + av[u][4] * xv[u][1] + av[u][5] * xv[u][2];
                acc[2] += av[u][6] * xv[u][0] + av[u][7] * xv[u][1] + av[u][8] * xv[u][2];
            }
        }
    }
}

// V selects the row product's shape: 0 three slots slot by slot, 1 three
// slots batched, 2 six slots batched (picked by the autotuner)
template <class T, int V>
__global__ void __launch_bounds__(256) k_sell_spmv(int nrows, const int* __restrict__ sp, const int* __restrict__ sci,
                                                   const T* __restrict__ S, const T* __restrict__ x,
                                                   T* __restrict__ y, const T* __restrict__ b, int mode,
                                                   const T* __restrict__ dinv, const double* __restrict__ scal) {
    pdl_trigger();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nrows) return;
    const int s = i >> 5, lane = i & 31;
    const int b0 = sp[s], w = (sp[s + 1] - b0) >> 5;
    const size_t sb = (size_t)(b0 >> 5);
    const int* cp = sci + b0 + lane;
    T acc[3] = {T(0), T(0), T(0)};
    sell_row_product<T, V == 2 ? 6 : 3, V != 0>(S, sb, lane, cp, w, x, acc);
    const T a0 = acc[0], a1 = acc[1], a2 = acc[2];
    const long o = 3L * i;
    if (mode == 0) { y[o] = a0; y[o + 1] = a1; y[o + 2] = a2; }
    else if (mode == 1) { y[o] = b[o] - a0; y[o + 1] = b[o + 1] - a1; y[o + 2] = b[o + 2] - a2; }
    else {
        const T sc = T(*scal);
        y[o] = sc * dinv[o] * a0; y[o + 1] = sc * dinv[o + 1] * a1; y[o + 2] = sc * dinv[o + 2] * a2;
    }
}

// fused Chebyshev step on the sliced-ELLPACK level-0 operator
template <class T, int V>
__global__ void __launch_bounds__(256) k_sell_cheb(int nrows, const int* __restrict__ sp, const int* __restrict__ sci,
                                                   const T* __restrict__ S, const T* __restrict__ dold,
                                                   T* __restrict__ dnew, T* __restrict__ r, T* __restrict__ x,
                                                   const T* __restrict__ dinv, const double* __restrict__ rho,
                                                   double cr, double cq) {
    pdl_trigger();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nrows) return;
    const int s = i >> 5, lane = i & 31;
    const int b0 = sp[s], w = (sp[s + 1] - b0) >> 5;
    const size_t sb = (size_t)(b0 >> 5);
    const int* cp = sci + b0 + lane;
    T t[3] = {T(0), T(0), T(0)};
    sell_row_product<T, V == 2 ? 6 : 3, V != 0>(S, sb, lane, cp, w, dold, t);
    const double delta = 0.5 * (*rho);
    const T c2 = T(cq / delta), c1 = T(cr);
#pragma unroll
    for (int q = 0; q < 3; q++) {
        const long o = 3L * i + q;
        const T rn = r[o] - t[q];
        const T dn = c1 * dold[o] + c2 * dinv[o] * rn;
        r[o] = rn;
        dnew[o] = dn;
        x[o] += dn;
    }
}

// ----------------------------------------------------------------- level 0 in FP16, diagonally scaled
// Mixed form: the level-0 smoother works on A^ = D^-1/2 A D^-1/2 (unit
// diagonal, |a^_ij| <= 1 for the SPD stiffness matrix) stored as FP16 in the
// sliced-ELLPACK layout, with hat variables x^ = D^1/2 x, b^ = D^-1/2 b,
// r^ = D^-1/2 r.  Chebyshev-Jacobi on A is Chebyshev on A^ with the identity
// there, so no diagonal is read; the matrix stream is 9 x 2 + 4 bytes per
// block instead of 9 x 4 + 4.  Arithmetic stays FP32.
__global__ void k_sell_half_build(int nrows, int nslices, const int* __restrict__ rp, const int* __restrict__ ci,
                                  const int* __restrict__ sp, const float* __restrict__ A,
                                  const float* __restrict__ dinv, __half* __restrict__ S) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = i >> 5, lane = i & 31;
    if (s >= nslices) return;
    const int base = sp[s] >> 5, w = (sp[s + 1] - sp[s]) >> 5;
    int r0 = 0, nb = 0;
    if (i < nrows) { r0 = rp[i]; nb = rp[i + 1] - r0; }
    float si[3] = {0.f, 0.f, 0.f};
    if (i < nrows)
        for (int q = 0; q < 3; q++) si[q] = sqrtf(fabsf(dinv[3L * i + q]));
    for (int k = 0; k < w; k++) {
        const int j = k < nb ? ci[r0 + k] : 0;
#pragma unroll
        for (int e = 0; e < 9; e++) {
            float v = 0.f;
            if (k < nb) v = A[(size_t)r0 * 9 + e * nb + k] * si[e / 3] * sqrtf(fabsf(dinv[3L * j + e % 3]));
            S[sell_idx<__half>(base + k, e, lane)] = __float2half_rn(v);
        }
    }
}
// s = D^1/2, sinv = D^-1/2 per DOF
__global__ void k_hat_scales(long n, const float* __restrict__ dinv, float* __restrict__ s, float* __restrict__ sinv) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const float d = fabsf(dinv[i]);
        sinv[i] = sqrtf(d);
        s[i] = d > 0.f ? 1.f / sqrtf(d) : 1.f;
    }
}
// MODE 1: y = b - A^ x          2: Chebyshev step t = A^ d; r -= t; d' = c1 d + c2 r; xo += d'
// MODE 3: y = sigma A^ x        4: y = s (b - A^ x)  (unscaled residual for the restriction)
template <int MODE>
__global__ void __launch_bounds__(256) k_sell_hat(int nrows, const int* __restrict__ sp, const int* __restrict__ sci,
                                                  const __half* __restrict__ S, const float* __restrict__ x,
                                                  float* __restrict__ y, const float* __restrict__ b,
                                                  float* __restrict__ r, float* __restrict__ xo,
                                                  const float* __restrict__ sc, const double* __restrict__ rho,
                                                  double cr, double cq) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nrows) return;
    const int s = i >> 5, lane = i & 31;
    const int b0 = sp[s], w = (sp[s + 1] - b0) >> 5;
    const size_t sb = (size_t)(b0 >> 5);
    const int* cp = sci + b0 + lane;
    float t0 = 0.f, t1 = 0.f, t2 = 0.f;
#pragma unroll 3
    for (int k = 0; k < w; k++) {
        const int j = __ldg(cp + 32 * k);
        const float x0 = x[3L * j], x1 = x[3L * j + 1], x2 = x[3L * j + 2];
        float av[9];
        sell_load9<__half>(S, sb + k, lane, av);
        t0 += av[0] * x0 + av[1] * x1 + av[2] * x2;
        t1 += av[3] * x0 + av[4] * x1 + av[5] * x2;
        t2 += av[6] * x0 + av[7] * x1 + av[8] * x2;
    }
    const float t[3] = {t0, t1, t2};
    const long o = 3L * i;
    if (MODE == 1) {
#pragma unroll
        for (int q = 0; q < 3; q++) y[o + q] = b[o + q] - t[q];
    } else if (MODE == 3) {
        const float sg = (float)(*rho);
#pragma unroll
        for (int q = 0; q < 3; q++) y[o + q] = sg * t[q];
    } else if (MODE == 4) {
#pragma unroll
        for (int q = 0; q < 3; q++) y[o + q] = sc[o + q] * (b[o + q] - t[q]);
    } else {
        const double delta = 0.5 * (*rho);
        const float c2 = (float)(cq / delta), c1 = (float)cr;
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const float rn = r[o + q] - t[q];
            const float dn = c1 * x[o + q] + c2 * rn;
            r[o + q] = rn;
            y[o + q] = dn;
            xo[o + q] += dn;
        }
    }
}
// first Chebyshev step on the hat variables (identity preconditioner)
__global__ void k_cheb_first_hat(long n, const float* __restrict__ b, float* __restrict__ r, float* __restrict__ d,
                                 float* __restrict__ x, const double* __restrict__ rho, int zero_init) {
    const float it = (float)(1.0 / (0.6 * (*rho)));
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        if (zero_init) {
            const float bi = b[i];
            r[i] = bi;
            d[i] = bi * it;
            x[i] = bi * it;
        } else {
            const float di = r[i] * it;
            d[i] = di;
            x[i] += di;
        }
    }
}
// b^ = D^-1/2 v (FP64 in, FP32 out) and x = D^-1/2 x^ in place
__global__ void k_to_hat(long n, const double* __restrict__ v, const float* __restrict__ sinv, float* __restrict__ b) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        b[i] = (float)(v[i] * (double)sinv[i]);
}
__global__ void k_from_hat(long n, const float* __restrict__ sinv, float* __restrict__ x) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) x[i] *= sinv[i];
}

// first Chebyshev step.  zero_init: r = b, d = Dinv b / theta, x = d.
// otherwise (r already = b - A x): d = Dinv r / theta, x += d.
template <class T>
__global__ void k_cheb_first(long n, const T* __restrict__ b, T* __restrict__ r, T* __restrict__ d, T* __restrict__ x,
                             const T* __restrict__ dinv, const double* __restrict__ rho, int zero_init) {
    pdl_trigger();
    const double theta = 0.6 * (*rho);
    const T it = T(1.0 / theta);
    pdl_wait();
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        if (zero_init) {
            T bi = b[i];
            r[i] = bi;
            T di = dinv[i] * bi * it;
            d[i] = di;
            x[i] = di;
        } else {
            T di = dinv[i] * r[i] * it;
            d[i] = di;
            x[i] += di;
        }
    }
}
// later Chebyshev step when A d was formed separately (element operator)
template <class T>
__global__ void k_cheb_upd(long n, const T* __restrict__ t, T* __restrict__ r, T* __restrict__ d, T* __restrict__ x,
                           const T* __restrict__ dinv, const double* __restrict__ rho, double cr, double cq) {
    const double delta = 0.5 * (*rho);
    const T c2 = T(cq / delta);
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        T rn = r[i] - t[i];
        T dn = T(cr) * d[i] + c2 * dinv[i] * rn;
        r[i] = rn;
        d[i] = dn;
        x[i] += dn;
    }
}

// ----------------------------------------------------------------- fixed-pattern SpGEMM
// entries of a BB-entry block stored block by block, rounded up to whole
// 16-byte vectors
template <class T, int BB>
__host__ __device__ constexpr int padded_block() {
    return (BB + 16 / (int)sizeof(T) - 1) / (16 / (int)sizeof(T)) * (16 / (int)sizeof(T));
}

// C = A * B with blocks A: BR x BK, B: BK x BC, C: BR x BC, from the
// product's plan (output-stationary): G lanes per C row, a lane owns one C block at a time and sums its contributing (A block,
// B block) pairs in registers: no shared memory, no atomics, no searches.
// BL 0: B slot-interleaved (the plan gives the block's first value), read
//       entry by entry; 1: B block by block, padded to 16-byte vectors (the
//       plan gives the block index), each block read as whole vectors.
// CL 0: C slot-interleaved, a row's entries written as coalesced runs;
//       1: C block by block, padded (the B operand of a later product).
template <class T, int BR, int BK, int BC, int GS, int PS, int BL, int CL>
__global__ void __launch_bounds__(256) k_spgemm_plan(int nrows, const int* __restrict__ Arp, const T* __restrict__ A,
                                                     const T* __restrict__ B, const int* __restrict__ Crp,
                                                     T* __restrict__ C, const int* __restrict__ pptr,
                                                     const uint2* __restrict__ pr) {
    // GS C blocks of a row at a time, each summed by PS lanes (long pair
    // lists: shorter dependent-load chains), combined by xor shuffles; the
    // next pair's plan entry is fetched while the current pair is summed
    constexpr int BRK = BR * BK, BKC = BK * BC, BRC = BR * BC, G = GS * PS;
    constexpr int VPL = 16 / (int)sizeof(T);
    constexpr int BKCP = padded_block<T, BKC>(), BRCP = padded_block<T, BRC>();
    const long tid = blockIdx.x * (long)blockDim.x + threadIdx.x;
    const int i = (int)(tid / G), gl = (int)(tid % G), gs = gl / PS, ps = gl % PS;
    if (i >= nrows) return;
    const unsigned lane = threadIdx.x & 31;
    const unsigned gmask = PS >= 32 ? 0xffffffffu : (((1u << PS) - 1u) << (lane & ~(unsigned)(PS - 1)));
    const int a0 = Arp[i], nA = Arp[i + 1] - a0;
    const int c0 = Crp[i], nC = Crp[i + 1] - c0;
    const T* Ar = A + (size_t)a0 * BRK;
    for (int sl = gs; sl < nC; sl += GS) {
        T acc[BRC];
#pragma unroll
        for (int e = 0; e < BRC; e++) acc[e] = T(0);
        const int p1 = pptr[c0 + sl + 1];
        int p = pptr[c0 + sl] + ps;
        uint2 w = p < p1 ? __ldg(pr + p) : make_uint2(0u, 0u);
        for (; p < p1; p += PS) {
            const int a = (int)(w.x >> 16), nB = (int)(w.x & 0xffffu);
            T ab[BRK], bb[BL ? BKCP : BKC];
#pragma unroll
            for (int e = 0; e < BRK; e++) ab[e] = __ldg(Ar + (size_t)e * nA + a);
            if constexpr (BL == 1) {
                const uint4* Bv = reinterpret_cast<const uint4*>(B + (size_t)w.y * BKCP);
#pragma unroll
                for (int q = 0; q < BKCP / VPL; q++) {
                    const uint4 t = __ldg(Bv + q);
                    memcpy(bb + q * VPL, &t, 16);
                }
            } else {
                const T* Bb = B + w.y;
#pragma unroll
                for (int e = 0; e < BKC; e++) bb[e] = __ldg(Bb + (size_t)e * nB);
            }
            if (p + PS < p1) w = __ldg(pr + p + PS);
#pragma unroll
            for (int r = 0; r < BR; r++)
#pragma unroll
                for (int cc = 0; cc < BC; cc++) {
                    T v = acc[r * BC + cc];
#pragma unroll
                    for (int m = 0; m < BK; m++) v += ab[r * BK + m] * bb[m * BC + cc];
                    acc[r * BC + cc] = v;
                }
        }
        if (PS > 1) {
#pragma unroll
            for (int e = 0; e < BRC; e++)
#pragma unroll
                for (int o = PS / 2; o > 0; o >>= 1) acc[e] += __shfl_xor_sync(gmask, acc[e], o);
        }
        if (ps == 0) {
            if constexpr (CL == 1) {
                T out[BRCP];
#pragma unroll
                for (int e = 0; e < BRC; e++) out[e] = acc[e];
#pragma unroll
                for (int e = BRC; e < BRCP; e++) out[e] = T(0);
                uint4* Cv = reinterpret_cast<uint4*>(C + (size_t)(c0 + sl) * BRCP);
#pragma unroll
                for (int q = 0; q < BRCP / VPL; q++) {
                    uint4 t;
                    memcpy(&t, out + q * VPL, 16);
                    Cv[q] = t;
                }
            } else {
#pragma unroll
                for (int e = 0; e < BRC; e++) C[(size_t)c0 * BRC + (size_t)e * nC + sl] = acc[e];
            }
        }
    }
}

// P block by block (padded to 16-byte vectors) from its slot-interleaved
// copy: warp per row, lanes over the row's values in storage order
template <class T, int BB>
__global__ void k_block_pad(int nrows, const int* __restrict__ rp, const T* __restrict__ P, T* __restrict__ Pb) {
    constexpr int BBP = padded_block<T, BB>();
    const int i = (int)((blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (i >= nrows) return;
    const int r0 = rp[i], nb = rp[i + 1] - r0;
    for (int t = lane; t < nb * BB; t += 32) {
        const int e = t / nb, sl = t - e * nb;
        Pb[(size_t)(r0 + sl) * BBP + e] = P[(size_t)r0 * BB + t];
    }
}

// P = Pt - (4 / (3 rho)) Dinv (A Pt), pattern of A Pt; Pt's block sits at ptpos
template <class T, int BS>
__global__ void k_smooth_p(int nnode, const int* __restrict__ rp, const int* __restrict__ ptpos,
                           const int* __restrict__ ptrp, const T* __restrict__ Ptv, const T* __restrict__ Tv,
                           const T* __restrict__ dinv, const double* __restrict__ rho, T* __restrict__ P,
                           T* __restrict__ Pb) {
    // P slot-interleaved, and block by block (padded) in Pb for the product A P
    constexpr int BB = BS * 6, BBP = padded_block<T, BB>();
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (i >= nnode) return;
    const T w = T(4.0 / (3.0 * (*rho)));
    const int r0 = rp[i], nb = rp[i + 1] - r0, pp = ptpos[i];
    const bool haspt = ptrp[i + 1] > ptrp[i];
    for (int q = lane; q < BB * nb; q += 32) {
        const int e = q / nb, s = q - e * nb, r = e / 6;
        T v = -w * dinv[(long)BS * i + r] * Tv[(size_t)r0 * BB + q];
        if (haspt && s == pp) v += Ptv[(size_t)ptrp[i] * BB + e];
        P[(size_t)r0 * BB + q] = v;
        Pb[(size_t)(r0 + s) * BBP + e] = v;
    }
}

// R = P^T (blocks 6 x BR from BR x 6), one warp per R row
template <class T, int BR>
__global__ void k_transpose(int nrows, const int* __restrict__ Rrp, const int* __restrict__ Rci,
                            const int* __restrict__ perm, const int* __restrict__ Prp, const T* __restrict__ P,
                            T* __restrict__ R) {
    constexpr int BB = 6 * BR;
    const int I = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (I >= nrows) return;
    const int r0 = Rrp[I], nb = Rrp[I + 1] - r0;
    for (int q = lane; q < BB * nb; q += 32) {
        const int e = q / nb, s = q - e * nb;
        const int a = e / BR, b = e % BR;
        const int j = Rci[r0 + s], pq = perm[r0 + s];
        const int pb = Prp[j], nbp = Prp[j + 1] - pb;
        R[(size_t)r0 * BB + q] = P[(size_t)pb * BB + (b * 6 + a) * nbp + (pq - pb)];
    }
}

// ----------------------------------------------------------------- power iteration / reductions
template <class T>
__global__ void k_dot2(long n, const T* __restrict__ v, const T* __restrict__ w, const double* __restrict__ scal,
                       double* __restrict__ part) {
    __shared__ double sm[64];
    double s[2] = {0.0, 0.0};
    const double sc = *scal;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        double wi = (double)w[i];
        s[0] += sc * (double)v[i] * wi;
        s[1] += wi * wi;
    }
    block_sum<2>(s, sm);
    if (threadIdx.x == 0) { part[2 * blockIdx.x] = s[0]; part[2 * blockIdx.x + 1] = s[1]; }
}
// lam = Rayleigh estimate, scal = 1/||w|| for the next step, cheb_rho =
// safety * lam (the Chebyshev smoother's spectral bound)
__global__ void k_power_final(int nb, const double* __restrict__ part, double* __restrict__ lam,
                              double* __restrict__ scal, double* __restrict__ cheb_rho, double safety) {
    __shared__ double sm[64];
    double s[2] = {0.0, 0.0};
    for (int i = threadIdx.x; i < nb; i += blockDim.x) { s[0] += part[2 * i]; s[1] += part[2 * i + 1]; }
    block_sum<2>(s, sm);
    if (threadIdx.x == 0) {
        *lam = s[0];
        *cheb_rho = safety * s[0];
        *scal = s[1] > 0.0 ? 1.0 / sqrt(s[1]) : 1.0;
    }
}
// start vector uniform in [-1, 1) from a splitmix64 hash of the index: rich
// in the high-frequency modes the power iteration must find
template <class T>
__global__ void k_power_seed(long n, T* __restrict__ v, double* __restrict__ scal) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        unsigned long long z = (unsigned long long)i * 0x9E3779B97F4A7C15ULL + 0x632BE59BD9B4E019ULL;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        z ^= z >> 31;
        v[i] = T(2.0 * (double)(z >> 11) * (1.0 / 9007199254740992.0) - 1.0);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *scal = 1.0 / sqrt((double)n / 3.0);
}

// ----------------------------------------------------------------- coarsest level
template <class T, int BS>
__global__ void k_bsr_to_dense(int nnode, const int* __restrict__ rp, const int* __restrict__ ci,
                               const T* __restrict__ A, double* __restrict__ M, int n) {
    const int i = blockIdx.x;
    if (i >= nnode) return;
    const int r0 = rp[i], nb = rp[i + 1] - r0;
    for (int q = threadIdx.x; q < BS * BS * nb; q += blockDim.x) {
        const int e = q / nb, s = q - e * nb, r = e / BS, cc = e % BS;
        const int j = ci[r0 + s];
        M[(size_t)(BS * i + r) * (2 * n) + BS * j + cc] = (double)A[(size_t)r0 * BS * BS + q];
    }
}
// [A | I] -> [I | A^-1] by Gauss-Jordan with partial pivoting, one CTA.
// A zero pivot (singular coarse operator) is replaced by 1 and flagged.
// When in_smem, [A | I] is staged in shared memory (n <= 112 fits in 227 KB):
// a single CTA is then bound by shared-memory rather than L2 bandwidth.
__global__ void k_gauss_jordan(int n, double* __restrict__ Mg, double* __restrict__ inv, int* __restrict__ flag,
                               int in_smem) {
    extern __shared__ double dyn[];  // n column factors [+ staged matrix]
    double* fk = dyn;
    __shared__ double s_val[32];
    __shared__ int s_idx[32];
    __shared__ double s_piv;
    __shared__ int s_prow;
    const int ld = 2 * n, tid = threadIdx.x, nt = blockDim.x;
    double* M = Mg;
    if (in_smem) {
        M = dyn + ((n + 1) & ~1);
        for (long q = tid; q < (long)n * ld; q += nt) M[q] = Mg[q];
    }
    __syncthreads();
    for (int q = tid; q < n; q += nt) M[(size_t)q * ld + n + q] = 1.0;
    __syncthreads();
    for (int k = 0; k < n; k++) {
        double best = -1.0;
        int bi = k;
        for (int i = k + tid; i < n; i += nt) {
            double v = fabs(M[(size_t)i * ld + k]);
            if (v > best) { best = v; bi = i; }
        }
        for (int o = 16; o > 0; o >>= 1) {
            double ov = __shfl_xor_sync(0xffffffffu, best, o);
            int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
        }
        if ((tid & 31) == 0) { s_val[tid >> 5] = best; s_idx[tid >> 5] = bi; }
        __syncthreads();
        if (tid == 0) {
            double bv = -1.0;
            int bidx = k;
            for (int w = 0; w < (nt + 31) / 32; w++)
                if (s_val[w] > bv || (s_val[w] == bv && s_idx[w] < bidx)) { bv = s_val[w]; bidx = s_idx[w]; }
            s_prow = bidx;
        }
        __syncthreads();
        const int pr = s_prow;
        if (pr != k)
            for (int j = tid; j < ld; j += nt) {
                double t = M[(size_t)k * ld + j];
                M[(size_t)k * ld + j] = M[(size_t)pr * ld + j];
                M[(size_t)pr * ld + j] = t;
            }
        __syncthreads();
        if (tid == 0) {
            double pv = M[(size_t)k * ld + k];
            if (pv == 0.0 || !isfinite(pv)) { pv = 1.0; *flag = 1; }
            s_piv = pv;
        }
        __syncthreads();
        const double ip = 1.0 / s_piv;
        for (int j = tid; j < ld; j += nt) M[(size_t)k * ld + j] *= ip;
        for (int i = tid; i < n; i += nt) fk[i] = M[(size_t)i * ld + k];
        __syncthreads();
        for (long q = tid; q < (long)n * ld; q += nt) {
            const int i = (int)(q / ld), j = (int)(q % ld);
            if (i != k) M[q] -= fk[i] * M[(size_t)k * ld + j];
        }
        __syncthreads();
    }
    for (long q = tid; q < (long)n * n; q += nt) {
        const int i = (int)(q / n), j = (int)(q % n);
        inv[q] = M[(size_t)i * ld + n + j];
    }
}
template <class T>
__global__ void k_dense_apply(int n, const double* __restrict__ inv, const T* __restrict__ b, T* __restrict__ x) {
    pdl_trigger();
    pdl_wait();
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (i >= n) return;
    double s = 0.0;
    for (int j = lane; j < n; j += 32) s += inv[(size_t)i * n + j] * (double)b[j];
    s = warp_sum(s);
    if (lane == 0) x[i] = T(s);
}

// the mixed form's FP64 right-hand side to FP32 and, on the same entries,
// the level-0 first Chebyshev step from the zero guess (the operations of
// k_cheb_first): r = b, d = x = Dinv b / (0.6 rho)
__global__ void k_convert_first(long n, const double* __restrict__ b64, float* __restrict__ b, float* __restrict__ r,
                                float* __restrict__ d, float* __restrict__ x, const float* __restrict__ dinv,
                                const double* __restrict__ rho) {
    const double theta = 0.6 * (*rho);
    const float it = float(1.0 / theta);
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const float bi = float(b64[i]);
        b[i] = bi;
        r[i] = bi;
        const float di = dinv[i] * bi * it;
        d[i] = di;
        x[i] = di;
    }
}
template <class TI, class TO>
__global__ void k_convert(long n, const TI* __restrict__ a, TO* __restrict__ b) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) b[i] = TO(a[i]);
}

// ----------------------------------------------------------------- coarse levels in one thread-block cluster
// The levels below l0 (a few thousand DOFs at most) are latency-bound: each
// of their sweeps is a tiny kernel.  One thread-block cluster (up to 16
// CTAs on 16 SMs) runs the whole lower part of the V-cycle from the
// restricted right-hand side at level l0 to the correction at level l0 --
// Chebyshev smoothing, residuals, restrictions, the dense coarsest solve and
// the prolongations, the same operations in the same order as the per-level
// kernels -- with hardware cluster barriers between the steps and every
// vector in global memory (L2-resident at these sizes).
template <class T>
struct CoarseArgs {
    int l0, L, deg_pre, deg_post;
    int nrow[kMaxLevels];                 // block rows (nodes) per level
    const int *Arp[kMaxLevels], *Aci[kMaxLevels], *Rrp[kMaxLevels], *Rci[kMaxLevels], *Prp[kMaxLevels],
        *Pci[kMaxLevels];
    const T *A[kMaxLevels], *R[kMaxLevels], *P[kMaxLevels], *dinv[kMaxLevels];
    T *x[kMaxLevels], *b[kMaxLevels], *r[kMaxLevels], *d[kMaxLevels], *d2[kMaxLevels], *t[kMaxLevels];
    const double* rho;                    // safety-scaled bounds, one per level
    const double* cinv;                   // coarsest dense inverse
    int ncoarse;
    double cr[16], cq[16];
};

__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ int cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return (int)r;
}
__device__ __forceinline__ int cluster_size() {
    uint32_t n;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(n));
    return (int)n;
}

// y = A x / y = b - A x / y += A x (mode 0/1/2) for 6x6 blocks over the cluster
template <class T>
__device__ __forceinline__ void cl_bsr66(int g0, int gs, int nrows, const int* __restrict__ rp,
                                         const int* __restrict__ ci, const T* __restrict__ A, const T* x, T* y,
                                         const T* b, int mode) {
    for (int o = g0; o < nrows * 6; o += gs) {
        const int row = o / 6, q = o - row * 6;
        const int r0 = rp[row], nb = rp[row + 1] - r0;
        const T* Ar = A + (size_t)r0 * 36;
        T s = T(0);
        for (int sl = 0; sl < nb; sl++) {
            const int j = ci[r0 + sl];
#pragma unroll
            for (int dd = 0; dd < 6; dd++) s += Ar[(size_t)(q * 6 + dd) * nb + sl] * x[6L * j + dd];
        }
        if (mode == 0) y[o] = s;
        else if (mode == 1) y[o] = b[o] - s;
        else y[o] += s;
    }
    cluster_sync_all();
}

template <class T>
__device__ void cl_smooth(const CoarseArgs<T>& a, int g0, int gs, int l, bool zero_init) {
    const int n = a.nrow[l] * 6;
    const T* dinv = a.dinv[l];
    T *x = a.x[l], *b = a.b[l], *r = a.r[l];
    T *dc = a.d[l], *dn = a.d2[l];
    const double rho = a.rho[l];
    const int deg = zero_init ? a.deg_pre : a.deg_post;
    if (!zero_init) cl_bsr66<T>(g0, gs, a.nrow[l], a.Arp[l], a.Aci[l], a.A[l], x, r, b, 1);
    const T it = T(1.0 / (0.6 * rho));
    for (int i = g0; i < n; i += gs) {
        if (zero_init) {
            const T bi = b[i];
            r[i] = bi;
            const T v = dinv[i] * bi * it;
            dc[i] = v;
            x[i] = v;
        } else {
            const T v = dinv[i] * r[i] * it;
            dc[i] = v;
            x[i] += v;
        }
    }
    cluster_sync_all();
    for (int k = 1; k < deg && k < 16; k++) {
        cl_bsr66<T>(g0, gs, a.nrow[l], a.Arp[l], a.Aci[l], a.A[l], dc, a.t[l], nullptr, 0);
        const T c2 = T(a.cq[k] / (0.5 * rho)), c1 = T(a.cr[k]);
        for (int i = g0; i < n; i += gs) {
            const T rn = r[i] - a.t[l][i];
            const T v = c1 * dc[i] + c2 * dinv[i] * rn;
            r[i] = rn;
            dn[i] = v;
            x[i] += v;
        }
        cluster_sync_all();
        T* tmp = dc;
        dc = dn;
        dn = tmp;
    }
}

// launched as exactly one cluster
template <class T>
__global__ void __launch_bounds__(512) k_coarse_cycle(CoarseArgs<T> a) {
    const int g0 = cluster_rank() * blockDim.x + threadIdx.x, gs = cluster_size() * blockDim.x;
    for (int l = a.l0; l < a.L; l++) {
        cl_smooth<T>(a, g0, gs, l, true);
        cl_bsr66<T>(g0, gs, a.nrow[l], a.Arp[l], a.Aci[l], a.A[l], a.x[l], a.t[l], a.b[l], 1);
        cl_bsr66<T>(g0, gs, a.nrow[l + 1], a.Rrp[l], a.Rci[l], a.R[l], a.t[l], a.b[l + 1], nullptr, 0);
    }
    {
        const int n = a.ncoarse;
        const T* bL = a.b[a.L];
        T* xL = a.x[a.L];
        for (int i = g0; i < n; i += gs) {
            double s = 0.0;
            for (int j = 0; j < n; j++) s += a.cinv[(size_t)i * n + j] * (double)bL[j];
            xL[i] = T(s);
        }
        cluster_sync_all();
    }
    for (int l = a.L - 1; l >= a.l0; l--) {
        cl_bsr66<T>(g0, gs, a.nrow[l], a.Prp[l], a.Pci[l], a.P[l], a.x[l + 1], a.x[l], nullptr, 2);
        cl_smooth<T>(a, g0, gs, l, false);
    }
}

// one cluster of up to 16 CTAs (8 where 16 cannot be co-scheduled)
template <class T>
static int launch_coarse_cycle(Ctx& c, const CoarseArgs<T>& a) {
    auto kern = k_coarse_cycle<T>;
    // cluster size that can be co-scheduled, found once per precision (threads
    // that race here compute the same value)
    static std::atomic<int> csize_cache[2] = {{0}, {0}};
    std::atomic<int>& csize_a = csize_cache[std::is_same<T, double>::value ? 1 : 0];
    int csize = csize_a.load(std::memory_order_relaxed);
    cudaLaunchConfig_t cfg{};
    cudaLaunchAttribute attr[1];
    cfg.blockDim = dim3(512, 1, 1);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = c.s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    if (csize == 0) {
        csize = 8;
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess) {
            int nclusters = 0;
            cfg.gridDim = dim3(16, 1, 1);
            attr[0].val.clusterDim.x = 16;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            if (cudaOccupancyMaxActiveClusters(&nclusters, kern, &cfg) == cudaSuccess && nclusters >= 1) csize = 16;
        }
        cudaGetLastError();
        csize_a.store(csize, std::memory_order_relaxed);
    }
    cfg.gridDim = dim3(csize, 1, 1);
    attr[0].val.clusterDim.x = csize;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    TCK(cudaLaunchKernelEx(&cfg, kern, a));
    note_launch();
    return 0;
}

// ----------------------------------------------------------------- host orchestration
template <class T>
static AmgVals<T>& vals(Ctx& c);
template <>
AmgVals<double>& vals<double>(Ctx& c) { return c.v64; }
template <>
AmgVals<float>& vals<float>(Ctx& c) { return c.v32; }

template <class T>
static int alloc_vals(Ctx& c) {
    AmgVals<T>& v = vals<T>(c);
    if (v.allocated) return 0;
    for (int l = 0; l < c.nlev; l++) {
        AmgDevLevel& D = c.dl[l];
        const int bs = D.bs;
        TRET(v.A[l].alloc((size_t)D.A.nnzb * bs * bs));
        TRET(v.dinv[l].alloc(D.ndof));
        TRET(v.x[l].alloc(D.ndof));
        TRET(v.b[l].alloc(D.ndof));
        TRET(v.r[l].alloc(D.ndof));
        TRET(v.d[l].alloc(D.ndof));
        TRET(v.d2[l].alloc(D.ndof));
        TRET(v.t[l].alloc(D.ndof));
        TRET(v.pv[l].alloc(D.ndof));
        TRET(v.pw[l].alloc(D.ndof));
        if (l == 0) {
            TRET(v.A0s.alloc((size_t)D.sell_blocks * 9));
            TRET(v.A0s.zero(c.s));  // padding slots are never written
        }
        if (l + 1 < c.nlev) {
            TRET(v.P[l].alloc((size_t)D.P.nnzb * bs * 6));
            TRET(v.T_[l].alloc((size_t)D.P.nnzb * bs * 6));
            // A P and the copy of P that is its B operand: block by block, padded
            const int bbp = bs == 3 ? padded_block<T, 18>() : padded_block<T, 36>();
            TRET(v.AP[l].alloc((size_t)D.AP.nnzb * bbp));
            TRET(v.AP[l].zero(c.s));
            TRET(v.Pb[l].alloc((size_t)D.P.nnzb * bbp));
            TRET(v.Pb[l].zero(c.s));
            TRET(v.R[l].alloc((size_t)D.R.nnzb * bs * 6));
            if (D.pnw) TRET(v.Pk[l].alloc((size_t)D.P.nnzb * bs * 6));
        }
        k_power_seed<T><<<grid_for(D.ndof, 256), 256, 0, c.s>>>(D.ndof, v.pv[l].p, c.rho.p + kMaxLevels + l), note_launch();
    }
    TCK(cudaGetLastError());
    v.allocated = true;
    return 0;
}

int amg_alloc(Ctx& c) {
    if (!c.rho.p) {
        TRET(c.rho.alloc(4 * kMaxLevels));
        TRET(c.rho.zero(c.s));
    }
    return 0;
}

template <class T>
static const T* pt_vals(Ctx& c, int l) {
    if (std::is_same<T, double>::value) return (const T*)c.dl[l].Pt64c.p;
    return (const T*)c.dl[l].Pt32c.p;
}
template <class T>
static const T* pt_vals_padded(Ctx& c, int l) {
    if (std::is_same<T, double>::value) return (const T*)c.dl[l].Pt64p.p;
    return (const T*)c.dl[l].Pt32p.p;
}

template <int BR, int BK, int BC, class T, int GS, int PS, int BL, int CL>
static void spgemm_plan_g(Ctx& c, const DevPattern& Ap, const T* A, const T* B, const DevPattern& Cp, T* C,
                          const ProductPlan& pl) {
    const long nt = (long)Cp.nrows * GS * PS;
    k_spgemm_plan<T, BR, BK, BC, GS, PS, BL, CL><<<(int)((nt + 255) / 256), 256, 0, c.s>>>(
        Cp.nrows, Ap.rp.p, A, B, Cp.rp.p, C, pl.ptr.p, pl.pr.p);
}
// C = A B from the product's plan: lanes per C block by the mean pair count,
// C blocks per row group by the mean row length (at most 32 lanes per row)
template <int BR, int BK, int BC, class T, int BL = 0, int CL = 0>
static int spgemm_plan(Ctx& c, const DevPattern& Ap, const T* A, const T* B, const DevPattern& Cp, T* C,
                       const ProductPlan& pl) {
    if (pl.avg_pairs >= 48) {
        if (pl.avg_row > 2) spgemm_plan_g<BR, BK, BC, T, 4, 8, BL, CL>(c, Ap, A, B, Cp, C, pl);
        else spgemm_plan_g<BR, BK, BC, T, 2, 8, BL, CL>(c, Ap, A, B, Cp, C, pl);
    } else if (pl.avg_pairs >= 16) {
        if (pl.avg_row > 4) spgemm_plan_g<BR, BK, BC, T, 8, 4, BL, CL>(c, Ap, A, B, Cp, C, pl);
        else spgemm_plan_g<BR, BK, BC, T, 4, 4, BL, CL>(c, Ap, A, B, Cp, C, pl);
    } else {
        if (pl.avg_row > 12) spgemm_plan_g<BR, BK, BC, T, 16, 1, BL, CL>(c, Ap, A, B, Cp, C, pl);
        else if (pl.avg_row > 6) spgemm_plan_g<BR, BK, BC, T, 8, 1, BL, CL>(c, Ap, A, B, Cp, C, pl);
        else spgemm_plan_g<BR, BK, BC, T, 4, 1, BL, CL>(c, Ap, A, B, Cp, C, pl);
    }
    note_launch();
    TCK(cudaGetLastError());
    return 0;
}

template <class T, int BR, int BC>
static int spmv(Ctx& c, const DevPattern& Ap, const T* A, const T* x, T* y, const T* b, int mode, const T* dinv = nullptr,
                const double* scal = nullptr, int gsel = 0, T* r5 = nullptr, T* d5 = nullptr, T* x5 = nullptr) {
    const long nrows = Ap.nrows;
    const double avg = nrows ? (double)Ap.nnzb / nrows : 1.0;
    int G = gsel;
    if (G != 8 && G != 16 && G != 32) G = avg <= 6.0 ? 8 : (avg <= 20.0 ? 16 : 32);
    if (G == 8) {
        TCK(launch_k(c.vc_pdl, k_bsr_spmv<T, BR, BC, 8>, dim3((unsigned)((nrows * 8 + 255) / 256)), dim3(256), 0, c.s,
                     (int)nrows, Ap.rp.p, Ap.ci.p, A, x, y, b, mode, dinv, scal, r5, d5, x5));
    } else if (G == 16) {
        TCK(launch_k(c.vc_pdl, k_bsr_spmv<T, BR, BC, 16>, dim3((unsigned)((nrows * 16 + 255) / 256)), dim3(256), 0, c.s,
                     (int)nrows, Ap.rp.p, Ap.ci.p, A, x, y, b, mode, dinv, scal, r5, d5, x5));
    } else {
        TCK(launch_k(c.vc_pdl, k_bsr_spmv<T, BR, BC, 32>, dim3((unsigned)((nrows * 32 + 255) / 256)), dim3(256), 0, c.s,
                     (int)nrows, Ap.rp.p, Ap.ci.p, A, x, y, b, mode, dinv, scal, r5, d5, x5));
    }
    TCK(cudaGetLastError());
    return 0;
}

// fused Chebyshev step on level l >= 1 with G lanes per block row
template <class T, int BS>
static int bsr_cheb(Ctx& c, int l, const T* dcur, T* dnxt, T* x, const double* rho, double cr, double cq) {
    AmgVals<T>& v = vals<T>(c);
    const AmgDevLevel& D = c.dl[l];
    const int nrows = D.nnode, G = c.tune.bsr_g[l];
    auto kern = G == 8 ? k_bsr_cheb<T, BS, 8> : (G == 16 ? k_bsr_cheb<T, BS, 16> : k_bsr_cheb<T, BS, 32>);
    const int g = (G == 8 || G == 16) ? G : 32;
    TCK(launch_k(c.vc_pdl, kern, dim3((unsigned)((nrows * g + 255) / 256)), dim3(256), 0, c.s, nrows, D.A.rp.p,
                 D.A.ci.p, v.A[l].p, dcur, dnxt, v.r[l].p, x, v.dinv[l].p, rho, cr, cq));
    return 0;
}

// P in the packed layout, after each numeric setup of P
template <class T>
static int pack_p(Ctx& c, int l) {
    AmgDevLevel& D = c.dl[l];
    AmgVals<T>& v = vals<T>(c);
    if (!D.pnw) return 0;
    const int grid = (int)(((long)D.P.nrows * 32 + 255) / 256);
    if (D.bs == 3)
        k_bsr_pack<T, 18><<<grid, 256, 0, c.s>>>(D.P.nrows, D.P.rp.p, v.P[l].p, v.Pk[l].p, D.P.nnzb), note_launch();
    else
        k_bsr_pack<T, 36><<<grid, 256, 0, c.s>>>(D.P.nrows, D.P.rp.p, v.P[l].p, v.Pk[l].p, D.P.nnzb), note_launch();
    TCK(cudaGetLastError());
    return 0;
}

// xf += P xc (mode 2) or xf += dinv (P xc) (mode 4)
template <class T>
static int prolong(Ctx& c, int l, const T* xc, T* xf, int mode, const T* dinv) {
    AmgDevLevel& D = c.dl[l];
    AmgVals<T>& v = vals<T>(c);
    if (D.pnw) {
        const int grid = (int)(((long)D.pnw * 32 + 255) / 256);
        if (D.bs == 3)
            TCK(launch_k(c.vc_pdl, k_bsr_lane<T, 3, 6>, dim3(grid), dim3(256), 0, c.s, D.pnw, D.pwrow.p, D.P.rp.p,
                         D.P.ci.p, v.Pk[l].p, D.P.nnzb, xc, xf, mode, dinv));
        else
            TCK(launch_k(c.vc_pdl, k_bsr_lane<T, 6, 6>, dim3(grid), dim3(256), 0, c.s, D.pnw, D.pwrow.p, D.P.rp.p,
                         D.P.ci.p, v.Pk[l].p, D.P.nnzb, xc, xf, mode, dinv));
        TCK(cudaGetLastError());
        return 0;
    }
    if (D.bs == 3) return spmv<T, 3, 6>(c, D.P, v.P[l].p, xc, xf, nullptr, mode, dinv);
    return spmv<T, 6, 6>(c, D.P, v.P[l].p, xc, xf, nullptr, mode, dinv);
}

// level 0 of the mixed form runs on the FP16 scaled operator (single load case)
static bool use_half0(const Ctx& c) {
    return c.p.precision == TOPO_PREC_MIXED && c.p.amg_half_fine && !c.p.fine_smoother_matfree &&
           !block_cases(c);
}
template <class T>
static bool half_level(const Ctx& c, int l) {
    return l == 0 && std::is_same<T, float>::value && use_half0(c) && c.h0.valid;
}
// hat-variable level-0 products (see k_sell_hat)
template <int MODE>
static int sell_hat(Ctx& c, const float* x, float* y, const float* b, float* r, float* xo, const float* sc,
                    const double* rho, double cr = 0.0, double cq = 0.0) {
    const AmgDevLevel& D = c.dl[0];
    k_sell_hat<MODE><<<(D.nnode + 255) / 256, 256, 0, c.s>>>(D.nnode, D.sell_ptr.p, D.sell_ci.p,
                                                             reinterpret_cast<const __half*>(c.h0.S.p), x, y, b, r, xo,
                                                             sc, rho, cr, cq), note_launch();
    TCK(cudaGetLastError());
    return 0;
}

template <class T>
static int level_spmv(Ctx& c, int l, const T* x, T* y, const T* b, int mode, const T* dinv = nullptr,
                      const double* scal = nullptr) {
    AmgVals<T>& v = vals<T>(c);
    if (half_level<T>(c, l) && (mode == 1 || mode == 3)) {
        // mode 1: r^ = b^ - A^ x^; mode 3: w = sigma A^ v (power iteration)
        const float* xf = reinterpret_cast<const float*>(x);
        float* yf = reinterpret_cast<float*>(y);
        cudaEvent_t e0;
        if (mode == 1) {
            prof_begin(c, PS_RES0, &e0);
            TRET(sell_hat<1>(c, xf, yf, reinterpret_cast<const float*>(b), nullptr, nullptr, nullptr, nullptr));
            prof_end(c, PS_RES0, e0);
        } else {
            TRET(sell_hat<3>(c, xf, yf, nullptr, nullptr, nullptr, nullptr, scal));
        }
        return 0;
    }
    if (l == 0 && mode != 2) {
        const AmgDevLevel& D = c.dl[0];
        cudaEvent_t e0;
        const bool rec = mode == 1;
        if (rec) prof_begin(c, PS_RES0, &e0);
        const int sb = c.tune.sell_block;
        const int sv = c.tune.sell_variant;
        TCK(launch_k(c.vc_pdl, sv == 2 ? k_sell_spmv<T, 2> : (sv == 1 ? k_sell_spmv<T, 1> : k_sell_spmv<T, 0>), dim3((D.nnode + sb - 1) / sb), dim3(sb), 0, c.s, D.nnode, D.sell_ptr.p,
                     D.sell_ci.p, v.A0s.p, x, y, b, mode, dinv, scal));
        if (rec) prof_end(c, PS_RES0, e0);
        TCK(cudaGetLastError());
        return 0;
    }
    if (c.dl[l].bs == 3) return spmv<T, 3, 3>(c, c.dl[l].A, v.A[l].p, x, y, b, mode, dinv, scal, c.tune.bsr_g[l]);
    return spmv<T, 6, 6>(c, c.dl[l].A, v.A[l].p, x, y, b, mode, dinv, scal, c.tune.bsr_g[l]);
}

template <class T>
static int estimate_rho(Ctx& c, int l, int iters) {
    AmgVals<T>& v = vals<T>(c);
    AmgDevLevel& D = c.dl[l];
    double* lam = c.rho.p + l;
    double* scal = c.rho.p + kMaxLevels + l;
    const int nb = grid_for(D.ndof, 256, 1024);
    if ((long)c.red.n < 2L * nb) TRET(c.red.alloc(std::max<long>(2L * nb, 4096)));
    for (int it = 0; it < iters; it++) {
        // w = sigma Dinv A v with sigma = 1/||v||; lam = (sigma v).w; sigma' = 1/||w||
        TRET(level_spmv<T>(c, l, v.pv[l].p, v.pw[l].p, (const T*)nullptr, 3, v.dinv[l].p, scal));
        k_dot2<T><<<nb, 256, 0, c.s>>>(D.ndof, v.pv[l].p, v.pw[l].p, scal, c.red.p), note_launch();
        k_power_final<<<1, 1024, 0, c.s>>>(nb, c.red.p, lam, scal, c.rho.p + 2 * kMaxLevels + l,
                                           c.p.cheb_safety > 0 ? c.p.cheb_safety : 1.0), note_launch();
        std::swap(v.pv[l], v.pw[l]);
    }
    TCK(cudaGetLastError());
    return 0;
}

template <class T>
static int numeric(Ctx& c) {
    TRET(alloc_vals<T>(c));
    AmgVals<T>& v = vals<T>(c);
    const T* ke = std::is_same<T, double>::value ? (const T*)c.ke64.p : (const T*)c.ke32.p;
    const T* Ee = std::is_same<T, double>::value ? (const T*)c.Ee64.p : (const T*)c.Ee32.p;
    cudaEvent_t pe;
    // level-0 assembly
    prof_begin(c, PS_SETUP_ASM, &pe);
    {
        AmgDevLevel& D = c.dl[0];
        const int wpb = 4;
        const size_t smem = (size_t)wpb * c.maxdeg * 9 * sizeof(T);
        const int grid = (c.nn + wpb - 1) / wpb;
        // the sliced-ELLPACK copy of the level-0 operator for the smoother is
        // written by the same pass (the mixed single-load form with the FP16
        // scaled copy built below does not need it)
        c.h0.valid = false;
        T* sell = (std::is_same<T, float>::value && use_half0(c)) ? nullptr : v.A0s.p;
        const long np = (long)c.n2e.n;
        if (!v.kst.p) {
            TRET(v.kst.alloc((size_t)np * 9 * c.nen));
            if (c.nen == 8)
                k_ke_node_rows<T, 8><<<grid_for(np * 72, 256), 256, 0, c.s>>>(np, c.n2e.p, ke, v.kst.p), note_launch();
            else
                k_ke_node_rows<T, 4><<<grid_for(np * 36, 256), 256, 0, c.s>>>(np, c.n2e.p, ke, v.kst.p), note_launch();
            TCK(cudaGetLastError());
        }
        if (c.nen == 8) {
            auto k = k_assemble_A0<T, 8>;
            TCK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            k<<<grid, wpb * 32, smem, c.s>>>(c.nn, c.n2e_ptr.p, c.n2e.p, c.bpos.p, v.kst.p, Ee, D.A.rp.p, D.A.ci.p,
                                              c.dof_fixed.p, v.A[0].p, c.maxdeg, sell, D.sell_ptr.p), note_launch();
        } else {
            auto k = k_assemble_A0<T, 4>;
            TCK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            k<<<grid, wpb * 32, smem, c.s>>>(c.nn, c.n2e_ptr.p, c.n2e.p, c.bpos.p, v.kst.p, Ee, D.A.rp.p, D.A.ci.p,
                                              c.dof_fixed.p, v.A[0].p, c.maxdeg, sell, D.sell_ptr.p), note_launch();
        }
        TCK(cudaGetLastError());
    }
    prof_end(c, PS_SETUP_ASM, pe);
    for (int l = 0; l < c.nlev; l++) {
        AmgDevLevel& D = c.dl[l];
        if (D.bs == 3)
            k_diag_inv<T, 3><<<grid_for(D.nnode, 256, 1 << 20), 256, 0, c.s>>>(D.nnode, D.A.rp.p, D.diagpos.p, v.A[l].p,
                                                                           v.dinv[l].p), note_launch();
        else
            k_diag_inv<T, 6><<<grid_for(D.nnode, 256, 1 << 20), 256, 0, c.s>>>(D.nnode, D.A.rp.p, D.diagpos.p, v.A[l].p,
                                                                           v.dinv[l].p), note_launch();
        TCK(cudaGetLastError());
        if (l == 0 && std::is_same<T, float>::value && use_half0(c)) {
            prof_begin(c, PS_SETUP_ASM, &pe);
            Half0& H = c.h0;
            if (!H.S.p) {
                TRET(H.S.alloc((size_t)D.sell_blocks * 9));
                TRET(H.s.alloc(D.ndof));
                TRET(H.sinv.alloc(D.ndof));
            }
            k_sell_half_build<<<D.nslices * 32 / 256 + 1, 256, 0, c.s>>>(
                D.nnode, D.nslices, D.A.rp.p, D.A.ci.p, D.sell_ptr.p, reinterpret_cast<const float*>(v.A[0].p),
                reinterpret_cast<const float*>(v.dinv[0].p), reinterpret_cast<__half*>(H.S.p)), note_launch();
            k_hat_scales<<<grid_for(D.ndof, 256), 256, 0, c.s>>>(D.ndof, reinterpret_cast<const float*>(v.dinv[0].p),
                                                                  H.s.p, H.sinv.p), note_launch();
            TCK(cudaGetLastError());
            H.valid = true;
            prof_end(c, PS_SETUP_ASM, pe);
        }
        if (l == c.nlev - 1) break;
        prof_begin(c, PS_SETUP_RHO, &pe);
        TRET(estimate_rho<T>(c, l, std::max(1, c.p.amg_rho_its)));
        prof_end(c, PS_SETUP_RHO, pe);
        prof_begin(c, PS_SETUP_GAL, &pe);
        AmgDevLevel& N = c.dl[l + 1];
        // T = A Pt ; P = Pt - w Dinv T
        const T* ptv = pt_vals<T>(c, l);
        if (D.bs == 3) {
            if (c.p.amg_smooth_p) {
                TRET((spgemm_plan<3, 3, 6, T, 1, 0>(c, D.A, v.A[l].p, pt_vals_padded<T>(c, l), D.P, v.T_[l].p, D.plan_T)));
                k_smooth_p<T, 3><<<(D.nnode * 32 + 255) / 256, 256, 0, c.s>>>(
                    D.nnode, D.P.rp.p, D.ptpos.p, D.Ptp.rp.p, ptv, v.T_[l].p, v.dinv[l].p, c.rho.p + l, v.P[l].p,
                    v.Pb[l].p), note_launch();
            } else {
                TCK(cudaMemcpyAsync(v.P[l].p, ptv, sizeof(T) * D.P.nnzb * 18, cudaMemcpyDeviceToDevice, c.s));
                k_block_pad<T, 18><<<(D.P.nrows * 32 + 255) / 256, 256, 0, c.s>>>(D.P.nrows, D.P.rp.p, v.P[l].p,
                                                                                  v.Pb[l].p), note_launch();
            }
            TRET((spgemm_plan<3, 3, 6, T, 1, 1>(c, D.A, v.A[l].p, v.Pb[l].p, D.AP, v.AP[l].p, D.plan_AP)));
            k_transpose<T, 3><<<(D.R.nrows * 32 + 255) / 256, 256, 0, c.s>>>(D.R.nrows, D.R.rp.p, D.R.ci.p, D.rperm.p,
                                                                             D.P.rp.p, v.P[l].p, v.R[l].p), note_launch();
            TRET((spgemm_plan<6, 3, 6, T, 1, 0>(c, D.R, v.R[l].p, v.AP[l].p, N.A, v.A[l + 1].p, D.plan_RAP)));
        } else {
            if (c.p.amg_smooth_p) {
                TRET((spgemm_plan<6, 6, 6, T, 1, 0>(c, D.A, v.A[l].p, pt_vals_padded<T>(c, l), D.P, v.T_[l].p, D.plan_T)));
                k_smooth_p<T, 6><<<(D.nnode * 32 + 255) / 256, 256, 0, c.s>>>(
                    D.nnode, D.P.rp.p, D.ptpos.p, D.Ptp.rp.p, ptv, v.T_[l].p, v.dinv[l].p, c.rho.p + l, v.P[l].p,
                    v.Pb[l].p), note_launch();
            } else {
                TCK(cudaMemcpyAsync(v.P[l].p, ptv, sizeof(T) * D.P.nnzb * 36, cudaMemcpyDeviceToDevice, c.s));
                k_block_pad<T, 36><<<(D.P.nrows * 32 + 255) / 256, 256, 0, c.s>>>(D.P.nrows, D.P.rp.p, v.P[l].p,
                                                                                  v.Pb[l].p), note_launch();
            }
            TRET((spgemm_plan<6, 6, 6, T, 1, 1>(c, D.A, v.A[l].p, v.Pb[l].p, D.AP, v.AP[l].p, D.plan_AP)));
            k_transpose<T, 6><<<(D.R.nrows * 32 + 255) / 256, 256, 0, c.s>>>(D.R.nrows, D.R.rp.p, D.R.ci.p, D.rperm.p,
                                                                             D.P.rp.p, v.P[l].p, v.R[l].p), note_launch();
            TRET((spgemm_plan<6, 6, 6, T, 1, 0>(c, D.R, v.R[l].p, v.AP[l].p, N.A, v.A[l + 1].p, D.plan_RAP)));
        }
        TRET(pack_p<T>(c, l));
        TCK(cudaGetLastError());
        prof_end(c, PS_SETUP_GAL, pe);
    }
    // coarsest: dense FP64 inverse
    prof_begin(c, PS_SETUP_COARSE, &pe);
    {
        const int L = c.nlev - 1;
        AmgDevLevel& D = c.dl[L];
        const int n = D.ndof;
        if (!c.cinv.p || (long)c.cinv.n < (long)n * n) {
            TRET(c.cinv.alloc((size_t)n * n));
            TRET(c.cA.alloc((size_t)n * 2 * n));
        }
        TCK(cudaMemsetAsync(c.cA.p, 0, sizeof(double) * (size_t)n * 2 * n, c.s));
        if (D.bs == 3)
            k_bsr_to_dense<T, 3><<<D.nnode, 128, 0, c.s>>>(D.nnode, D.A.rp.p, D.A.ci.p, v.A[L].p, c.cA.p, n), note_launch();
        else
            k_bsr_to_dense<T, 6><<<D.nnode, 128, 0, c.s>>>(D.nnode, D.A.rp.p, D.A.ci.p, v.A[L].p, c.cA.p, n), note_launch();
        const size_t smg = sizeof(double) * (size_t)(((n + 1) & ~1) + (size_t)2 * n * n);
        const int in_smem = smg <= 220 * 1024;
        const size_t sm = in_smem ? smg : sizeof(double) * (size_t)n;
        if (sm > 48 * 1024) TCK(cudaFuncSetAttribute(k_gauss_jordan, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_gauss_jordan<<<1, 1024, sm, c.s>>>(n, c.cA.p, c.cinv.p, reinterpret_cast<int*>(c.rho.p + 3 * kMaxLevels),
                                             in_smem), note_launch();
        TCK(cudaGetLastError());
    }
    prof_end(c, PS_SETUP_COARSE, pe);
    return 0;
}

// Chebyshev recurrence numbers for sigma = theta/delta = 1.2
void cheb_coeffs(int deg, double* cr, double* cq) {
    const double sigma = 1.2;
    double rho_prev = 1.0 / sigma;
    for (int k = 1; k < deg; k++) {
        double rk = 1.0 / (2.0 * sigma - rho_prev);
        cr[k] = rk * rho_prev;
        cq[k] = 2.0 * rk;
        rho_prev = rk;
    }
}

template <class T>
// first_done: the first Chebyshev step from the zero guess (r = b,
// d = x = Dinv b / theta) was already taken by the kernel that produced b
static int smooth(Ctx& c, int l, const T* b, T* x, bool zero_init, bool first_done = false) {
    AmgVals<T>& v = vals<T>(c);
    AmgDevLevel& D = c.dl[l];
    const long n = D.ndof;
    // pre-smoothing (zero initial guess) and post-smoothing degrees
    int deg = (!zero_init && c.p.cheb_degree_post > 0) ? c.p.cheb_degree_post : c.p.cheb_degree;
    if (l > 0 && c.p.cheb_degree_coarse > 0) deg = c.p.cheb_degree_coarse;  // levels below the finest
    deg = std::max(1, deg);
    double cr[16] = {0}, cq[16] = {0};
    cheb_coeffs(std::min(deg, 16), cr, cq);
    const double* rho = c.rho.p + 2 * kMaxLevels + l;  // safety-scaled spectral bound
    if (half_level<T>(c, l)) {
        // Chebyshev on A^ in hat variables: no diagonal
        float* xf = reinterpret_cast<float*>(x);
        const float* bf = reinterpret_cast<const float*>(b);
        float* r = reinterpret_cast<float*>(v.r[0].p);
        float* dc = reinterpret_cast<float*>(v.d[0].p);
        float* dn = reinterpret_cast<float*>(v.d2[0].p);
        if (!zero_init) TRET(level_spmv<T>(c, 0, x, v.r[0].p, b, 1));
        k_cheb_first_hat<<<grid_for(n, 256), 256, 0, c.s>>>(n, bf, r, dc, xf, rho, zero_init ? 1 : 0), note_launch();
        for (int k = 1; k < deg && k < 16; k++) {
            cudaEvent_t e0;
            prof_begin(c, PS_CHEB0, &e0);
            TRET(sell_hat<2>(c, dc, dn, nullptr, r, xf, nullptr, rho, cr[k], cq[k]));
            prof_end(c, PS_CHEB0, e0);
            std::swap(dc, dn);
        }
        TCK(cudaGetLastError());
        return 0;
    }
    const bool matfree = (l == 0) && c.p.fine_smoother_matfree;
    if (!zero_init) {
        // r = b - A x
        if (matfree) {
            if (std::is_same<T, float>::value) TRET(kmatvec32(c, (const float*)x, (float*)v.r[l].p, (const float*)b));
            else TRET(kmatvec64r(c, (const double*)x, (double*)v.r[l].p, (const double*)b));
        } else {
            TRET(level_spmv<T>(c, l, x, v.r[l].p, b, 1));
        }
    }
    if (!(zero_init && first_done))
        TCK(launch_k(c.vc_pdl, k_cheb_first<T>, dim3(grid_for(n, 256)), dim3(256), 0, c.s, n, b, v.r[l].p, v.d[l].p, x,
                     v.dinv[l].p, rho, zero_init ? 1 : 0));
    T* dcur = v.d[l].p;
    T* dnxt = v.d2[l].p;
    for (int k = 1; k < deg && k < 16; k++) {
        if (matfree) {
            if (std::is_same<T, float>::value) TRET(kmatvec32(c, (const float*)dcur, (float*)v.t[l].p, nullptr));
            else TRET(kmatvec64r(c, (const double*)dcur, (double*)v.t[l].p, nullptr));
            k_cheb_upd<T><<<grid_for(n, 256), 256, 0, c.s>>>(n, v.t[l].p, v.r[l].p, dcur, x, v.dinv[l].p, rho, cr[k], cq[k]), note_launch();
        } else {
            const int nrows = D.nnode;
            if (l == 0) {
                cudaEvent_t e0;
                prof_begin(c, PS_CHEB0, &e0);
                const int sv = c.tune.sell_variant;
                TCK(launch_k(c.vc_pdl, sv == 2 ? k_sell_cheb<T, 2> : (sv == 1 ? k_sell_cheb<T, 1> : k_sell_cheb<T, 0>), dim3((nrows + c.tune.sell_block - 1) / c.tune.sell_block),
                             dim3(c.tune.sell_block), 0, c.s, nrows, D.sell_ptr.p, D.sell_ci.p, v.A0s.p, dcur, dnxt,
                             v.r[l].p, x, v.dinv[l].p, rho, cr[k], cq[k]));
                prof_end(c, PS_CHEB0, e0);
            } else if (D.bs == 3) {
                TRET((bsr_cheb<T, 3>(c, l, dcur, dnxt, x, rho, cr[k], cq[k])));
            } else {
                TRET((bsr_cheb<T, 6>(c, l, dcur, dnxt, x, rho, cr[k], cq[k])));
            }
            std::swap(dcur, dnxt);
        }
        TCK(cudaGetLastError());
    }
    return 0;
}

// first level (>= 1) small enough for the one-cluster lower V-cycle, or -1
static int coarse_cta_level(const Ctx& c) {
    if (!c.p.amg_coarse_cta) return -1;
    for (int l = 1; l < c.nlev; l++)
        if (c.dl[l].bs == 6 && (long)c.dl[l].ndof <= 8192) return l;
    return -1;
}

// V-cycle launches use programmatic dependent launch while one is in flight
struct PdlScope {
    Ctx& c;
    PdlScope(Ctx& cc, bool on) : c(cc) { c.vc_pdl = on; }
    ~PdlScope() { c.vc_pdl = false; }
};

template <class T>
// first0_done: the level-0 first Chebyshev step was taken with the
// right-hand side's conversion (k_convert_first)
static int vcycle(Ctx& c, const T* b0, T* x0, bool first0_done = false) {
    PdlScope pdl_scope(c, c.p.pdl != 0);
    AmgVals<T>& v = vals<T>(c);
    const int L = c.nlev - 1;
    const T* bl[kMaxLevels];
    T* xl[kMaxLevels];
    for (int l = 0; l <= L; l++) { bl[l] = v.b[l].p; xl[l] = v.x[l].p; }
    bl[0] = b0;
    xl[0] = x0;
    cudaEvent_t ecoarse = nullptr;
    // levels l0..L run in one CTA (k_coarse_cycle); above them, per-level kernels
    const int l0 = coarse_cta_level(c);
    const int ldown = l0 > 0 ? l0 : L;
    bool first_done = first0_done && !half_level<T>(c, 0);
    for (int l = 0; l < ldown; l++) {
        AmgDevLevel& D = c.dl[l];
        TRET(smooth<T>(c, l, bl[l], xl[l], true, first_done));
        if (half_level<T>(c, l)) {
            // unscaled residual t = D^1/2 (b^ - A^ x^) for the restriction
            cudaEvent_t e0;
            prof_begin(c, PS_RES0, &e0);
            TRET(sell_hat<4>(c, reinterpret_cast<const float*>(xl[0]), reinterpret_cast<float*>(v.t[0].p),
                             reinterpret_cast<const float*>(bl[0]), nullptr, nullptr, c.h0.s.p, nullptr));
            prof_end(c, PS_RES0, e0);
        } else if (l == 0 && c.p.fine_smoother_matfree) {
            if (std::is_same<T, float>::value) TRET(kmatvec32(c, (const float*)xl[0], (float*)v.t[0].p, (const float*)bl[0]));
            else TRET(kmatvec64r(c, (const double*)xl[0], (double*)v.t[0].p, (const double*)bl[0]));
        } else {
            TRET(level_spmv<T>(c, l, xl[l], v.t[l].p, bl[l], 1));
        }
        // when level l+1 is smoothed next, its first step from the zero guess
        // is taken by the restriction that produces its right-hand side
        const bool fuse = l + 1 < ldown;
        const int rmode = fuse ? 5 : 0;
        const T* di5 = fuse ? v.dinv[l + 1].p : nullptr;
        const double* rho5 = fuse ? c.rho.p + 2 * kMaxLevels + l + 1 : nullptr;
        T* r5 = fuse ? v.r[l + 1].p : nullptr;
        T* d5 = fuse ? v.d[l + 1].p : nullptr;
        T* x5 = fuse ? xl[l + 1] : nullptr;
        if (D.bs == 3)
            TRET((spmv<T, 6, 3>(c, D.R, v.R[l].p, v.t[l].p, v.b[l + 1].p, nullptr, rmode, di5, rho5, 0, r5, d5, x5)));
        else
            TRET((spmv<T, 6, 6>(c, D.R, v.R[l].p, v.t[l].p, v.b[l + 1].p, nullptr, rmode, di5, rho5, 0, r5, d5, x5)));
        first_done = fuse;
        if (l == 0) prof_begin(c, PS_VC_COARSE, &ecoarse);
    }
    if (l0 > 0) {
        CoarseArgs<T> a{};
        a.l0 = l0;
        a.L = L;
        const int dc = c.p.cheb_degree_coarse;
        a.deg_pre = std::max(1, dc > 0 ? dc : c.p.cheb_degree);
        a.deg_post = std::max(1, dc > 0 ? dc : (c.p.cheb_degree_post > 0 ? c.p.cheb_degree_post : c.p.cheb_degree));
        for (int l = l0; l <= L; l++) {
            AmgDevLevel& D = c.dl[l];
            a.nrow[l] = D.nnode;
            a.Arp[l] = D.A.rp.p;
            a.Aci[l] = D.A.ci.p;
            a.A[l] = v.A[l].p;
            a.dinv[l] = v.dinv[l].p;
            a.x[l] = v.x[l].p;
            a.b[l] = v.b[l].p;
            a.r[l] = v.r[l].p;
            a.d[l] = v.d[l].p;
            a.d2[l] = v.d2[l].p;
            a.t[l] = v.t[l].p;
            if (l < L) {
                a.Rrp[l] = D.R.rp.p;
                a.Rci[l] = D.R.ci.p;
                a.R[l] = v.R[l].p;
                a.Prp[l] = D.P.rp.p;
                a.Pci[l] = D.P.ci.p;
                a.P[l] = v.P[l].p;
            }
        }
        a.rho = c.rho.p + 2 * kMaxLevels;
        a.cinv = c.cinv.p;
        a.ncoarse = c.dl[L].ndof;
        cheb_coeffs(16, a.cr, a.cq);
        TRET(launch_coarse_cycle<T>(c, a));
    } else {
        const int n = c.dl[L].ndof;
        TCK(launch_k(c.vc_pdl, k_dense_apply<T>, dim3((n * 32 + 255) / 256), dim3(256), 0, c.s, n, c.cinv.p, v.b[L].p,
                     v.x[L].p));
        TCK(cudaGetLastError());
    }
    for (int l = ldown - 1; l >= 0; l--) {
        if (l == 0) prof_end(c, PS_VC_COARSE, ecoarse);
        if (half_level<T>(c, l))  // x^ += D^1/2 P e
            TRET(prolong<T>(c, l, v.x[l + 1].p, xl[l], 4, reinterpret_cast<const T*>(c.h0.s.p)));
        else
            TRET(prolong<T>(c, l, v.x[l + 1].p, xl[l], 2, nullptr));
        TRET(smooth<T>(c, l, bl[l], xl[l], false));
    }
    if (half_level<T>(c, 0)) {
        const long n0 = c.dl[0].ndof;
        k_from_hat<<<grid_for(n0, 256), 256, 0, c.s>>>(n0, c.h0.sinv.p, reinterpret_cast<float*>(x0)), note_launch();
        TCK(cudaGetLastError());
    }
    return 0;
}

// re-seed the warm-started power iterations (a fresh optimisation run then
// reproduces the first one's preconditioners)
template <class T>
static int reseed(Ctx& c) {
    AmgVals<T>& v = vals<T>(c);
    if (!v.allocated) return 0;
    for (int l = 0; l < c.nlev; l++) {
        k_power_seed<T><<<grid_for(c.dl[l].ndof, 256), 256, 0, c.s>>>(c.dl[l].ndof, v.pv[l].p, c.rho.p + kMaxLevels + l),
            note_launch();
    }
    TCK(cudaGetLastError());
    return 0;
}
int amg_reset_warm_start(Ctx& c) {
    TRET(reseed<double>(c));
    return reseed<float>(c);
}

// host copy of level l matrix `which` (0 A, 1 P, 2 R) as plain BSR
template <class T>
static int level_copy(Ctx& c, int l, int which, std::vector<double>& out, const DevPattern*& pat, int& br, int& bc) {
    AmgVals<T>& v = vals<T>(c);
    if (!v.allocated) { set_error("no AMG hierarchy built yet (run a solve first)"); return TOPO_ERR_ARG; }
    const AmgDevLevel& D = c.dl[l];
    const T* src;
    if (which == 0) { pat = &D.A; br = bc = D.bs; src = v.A[l].p; }
    else if (which == 1) { pat = &D.P; br = D.bs; bc = 6; src = v.P[l].p; }
    else { pat = &D.R; br = 6; bc = D.bs; src = v.R[l].p; }
    const long nv = pat->nnzb * br * bc;
    std::vector<T> raw(nv);
    std::vector<int> rp(pat->nrows + 1);
    TCK(cudaMemcpyAsync(raw.data(), src, sizeof(T) * nv, cudaMemcpyDeviceToHost, c.s));
    TCK(cudaMemcpyAsync(rp.data(), pat->rp.p, sizeof(int) * (pat->nrows + 1), cudaMemcpyDeviceToHost, c.s));
    TCK(cudaStreamSynchronize(c.s));
    out.assign(nv, 0.0);
    const int bb = br * bc;
    for (int i = 0; i < pat->nrows; i++) {
        const int r0 = rp[i], nb = rp[i + 1] - r0;
        for (int s = 0; s < nb; s++)
            for (int e = 0; e < bb; e++) out[((size_t)r0 + s) * bb + e] = (double)raw[(size_t)r0 * bb + e * nb + s];
    }
    return 0;
}

int amg_level_copy(Ctx& c, int l, int which, std::vector<double>& vals_out, std::vector<int>& rp, std::vector<int>& ci,
                   int& nrows, int& ncols, int& br, int& bc) {
    if (l < 0 || l >= c.nlev || which < 0 || which > 2 || (which > 0 && l == c.nlev - 1)) {
        set_error("no such AMG level matrix");
        return TOPO_ERR_ARG;
    }
    const DevPattern* pat = nullptr;
    if (c.p.precision == TOPO_PREC_MIXED) TRET(level_copy<float>(c, l, which, vals_out, pat, br, bc));
    else TRET(level_copy<double>(c, l, which, vals_out, pat, br, bc));
    nrows = pat->nrows;
    ncols = pat->ncols;
    rp.resize(nrows + 1);
    ci.resize(pat->nnzb);
    TCK(cudaMemcpy(rp.data(), pat->rp.p, sizeof(int) * (nrows + 1), cudaMemcpyDeviceToHost));
    TCK(cudaMemcpy(ci.data(), pat->ci.p, sizeof(int) * pat->nnzb, cudaMemcpyDeviceToHost));
    return 0;
}

// y = A0 x with the level-0 smoother's operator (sliced ELLPACK, current
// precision); -1 when the FP16 scaled copy replaces it.  Used to time launch
// shapes.
int amg_level0_apply(Ctx& c, const void* x, void* y) {
    if (c.p.precision == TOPO_PREC_MIXED) {
        if (half_level<float>(c, 0) || !c.v32.allocated) return -1;
        return level_spmv<float>(c, 0, static_cast<const float*>(x), static_cast<float*>(y), nullptr, 0);
    }
    if (!c.v64.allocated) return -1;
    return level_spmv<double>(c, 0, static_cast<const double*>(x), static_cast<double*>(y), nullptr, 0);
}

// Lanes per block row (8, 16 or 32) of the smoothing and residual products
// on each level >= 1 that is smoothed, timed (best of 3 runs of 8 back-to-back
// launches, CUDA events) as the residual t = b - A x on the current
// hierarchy's own matrices.
template <class T>
static int tune_levels(Ctx& c) {
    AmgVals<T>& v = vals<T>(c);
    if (!v.allocated) return 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    TCK(cudaEventCreate(&e0));
    TCK(cudaEventCreate(&e1));
    int rc = 0;
    for (int l = 1; l + 1 < c.nlev && rc == 0; l++) {
        float best = 1e30f;
        int pick = 0;
        for (int g : {8, 16, 32}) {
            c.tune.bsr_g[l] = g;
            for (int rep = 0; rep < 3 && rc == 0; rep++) {
                float t = 0.f;
                if (cudaEventRecord(e0, c.s) != cudaSuccess) { rc = TOPO_ERR_CUDA; break; }
                for (int it = 0; it < 8 && rc == 0; it++) rc = level_spmv<T>(c, l, v.x[l].p, v.t[l].p, v.b[l].p, 1);
                if (rc == 0 && (cudaEventRecord(e1, c.s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                                cudaEventElapsedTime(&t, e0, e1) != cudaSuccess))
                    rc = TOPO_ERR_CUDA;
                if (rc == 0 && t < best) { best = t; pick = g; }
            }
        }
        c.tune.bsr_g[l] = pick;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != 0) {
        cudaGetLastError();
        for (int l = 0; l < kMaxLevels; l++) c.tune.bsr_g[l] = 0;
        set_error("AMG level tuning failed");
    }
    return rc;
}

int amg_tune_levels(Ctx& c) {
    if (c.nlev < 3) return 0;
    if (c.p.precision == TOPO_PREC_MIXED) return tune_levels<float>(c);
    return tune_levels<double>(c);
}

int amg_numeric(Ctx& c) {
    TRET(amg_alloc(c));
    if (c.p.precision == TOPO_PREC_MIXED) return numeric<float>(c);
    return numeric<double>(c);
}

int amg_vcycle64(Ctx& c, const double* b, double* x) { return vcycle<double>(c, b, x); }

int amg_vcycle32(Ctx& c, const double* b64, float* x) {
    AmgVals<float>& v = c.v32;
    const long n = c.dl[0].ndof;
    const bool half = half_level<float>(c, 0);
    if (half)
        k_to_hat<<<grid_for(n, 256), 256, 0, c.s>>>(n, b64, c.h0.sinv.p, v.b[0].p), note_launch();
    else
        k_convert_first<<<grid_for(n, 256), 256, 0, c.s>>>(n, b64, v.b[0].p, v.r[0].p, v.d[0].p, x, v.dinv[0].p,
                                                          c.rho.p + 2 * kMaxLevels), note_launch();
    TCK(cudaGetLastError());
    // level-0 rhs lives in v.b[0]; the smoother keeps b intact
    return vcycle<float>(c, v.b[0].p, x, !half);
}

}  // namespace topo
