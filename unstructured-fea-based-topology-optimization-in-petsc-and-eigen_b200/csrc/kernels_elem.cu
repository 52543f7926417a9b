// kernels_elem.cu -- element-level sm_100a kernels: element matrices (once per
// mesh), the matrix-free SIMP operator K(x) u, compliance/sensitivity
// reductions, the Helmholtz-filter operators and the von Mises stress.
//
// Layout: element data live in AoSoA tiles of 32 elements -- entry k of the
// element in lane l of tile t sits at base[(t*NK + k)*32 + l] -- so a warp
// that owns one tile (one element per lane) reads every entry of its 32
// element matrices as one coalesced 256-byte (FP64) / 128-byte (FP32) line.
#include <cuda_runtime.h>

#include "ctx.h"

namespace topo {

// ----------------------------------------------------------------- element geometry
// rounded 3-point Gauss rule of the reference (SolveFem.cpp:364-365,
// PDEFilter.cpp:195-196)
__constant__ double c_gp[3] = {-0.775, 0.0, 0.775};
__constant__ double c_gw[3] = {0.556, 0.889, 0.556};

__device__ __forceinline__ double inv3(const double J[9], double Ji[9]) {
    double c00 = J[4] * J[8] - J[5] * J[7];
    double c01 = J[5] * J[6] - J[3] * J[8];
    double c02 = J[3] * J[7] - J[4] * J[6];
    double det = J[0] * c00 + J[1] * c01 + J[2] * c02;
    double id = 1.0 / det;
    Ji[0] = c00 * id;
    Ji[1] = (J[2] * J[7] - J[1] * J[8]) * id;
    Ji[2] = (J[1] * J[5] - J[2] * J[4]) * id;
    Ji[3] = c01 * id;
    Ji[4] = (J[0] * J[8] - J[2] * J[6]) * id;
    Ji[5] = (J[2] * J[3] - J[0] * J[5]) * id;
    Ji[6] = c02 * id;
    Ji[7] = (J[1] * J[6] - J[0] * J[7]) * id;
    Ji[8] = (J[0] * J[4] - J[1] * J[3]) * id;
    return det;
}

__device__ __forceinline__ double det3v(const double* a, const double* b, const double* c) {
    return a[0] * (b[1] * c[2] - b[2] * c[1]) - a[1] * (b[0] * c[2] - b[2] * c[0]) + a[2] * (b[0] * c[1] - b[1] * c[0]);
}

// decode packed upper-triangular index k of an n x n matrix into (i, j), i <= j
__device__ __forceinline__ void unpack_ij(int k, int n, int& i, int& j) {
    int row = 0, len = n;
    while (k >= len) { k -= len; row++; len--; }
    i = row;
    j = row + k;
}
__host__ __device__ __forceinline__ int pk_index(int i, int j, int n) {
    if (i > j) { int t = i; i = j; j = t; }
    return i * n - (i * (i - 1)) / 2 + (j - i);
}

// Element matrices of one hex8 element per warp: the 300 packed entries of Ke
// (E = 1, SolveFem::Hex8Isoparametric), the 36 packed entries of the Helmholtz
// matrix and the 8 entries of T (PDEFilter::KeHel), and the 5-tet volume
// (SolveFem::ComputeVolOfHex).  All lanes evaluate the 27 Gauss points; each
// lane accumulates its own packed entries.  Stiffness entries use the
// isotropic closed form of B'DB: for DOFs (ci,li),(cj,lj)
//   lam dN_ci,li dN_cj,lj + mu dN_cj,li dN_ci,lj + mu [ci==cj] grad N_li . grad N_lj.
__global__ void k_hex8_setup(int ne, const int* __restrict__ elem, const double* __restrict__ vertex, double nu,
                             double rmin, double* __restrict__ ke64, float* __restrict__ ke32,
                             double* __restrict__ vol, double* __restrict__ kf, double* __restrict__ tf) {
    const int e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (e >= ne) return;
    const int tile = e >> 5, el = e & 31;
    double co[24];
#pragma unroll
    for (int l = 0; l < 8; l++) {
        int nd = elem[(long)e * 8 + l];
#pragma unroll
        for (int q = 0; q < 3; q++) co[3 * l + q] = vertex[3L * nd + q];
    }
    const double lam = nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double mu = 1.0 / (2.0 * (1.0 + nu));
    const double r = 1.0 / (2.0 * sqrt(3.0)) * rmin;
    const double r2 = r * r;
    int ci[10], li[10], cj[10], lj[10];
    double acc[10];
#pragma unroll
    for (int t = 0; t < 10; t++) {
        int k = lane + 32 * t, i = 0, j = 0;
        if (k < 300) unpack_ij(k, 24, i, j);
        ci[t] = i / 8; li[t] = i % 8; cj[t] = j / 8; lj[t] = j % 8;
        acc[t] = 0.0;
    }
    int fi[2], fj[2];
    double facc[2] = {0.0, 0.0}, tacc = 0.0;
#pragma unroll
    for (int t = 0; t < 2; t++) {
        int k = lane + 32 * t, i = 0, j = 0;
        if (k < 36) unpack_ij(k, 8, i, j);
        fi[t] = i; fj[t] = j;
    }
    for (int g = 0; g < 27; g++) {
        const double xi = c_gp[g / 9], eta = c_gp[(g / 3) % 3], zeta = c_gp[g % 3];
        const double w = c_gw[g / 9] * c_gw[(g / 3) % 3] * c_gw[g % 3];
        double Nd[24], N[8];
#pragma unroll
        for (int l = 0; l < 8; l++) {
            double sa = (l & 1) ? 1.0 : -1.0, sb = (l & 2) ? 1.0 : -1.0, sc = (l & 4) ? 1.0 : -1.0;
            Nd[l] = 0.125 * sa * (1.0 + sb * eta) * (1.0 + sc * zeta);
            Nd[8 + l] = 0.125 * sb * (1.0 + sa * xi) * (1.0 + sc * zeta);
            Nd[16 + l] = 0.125 * sc * (1.0 + sa * xi) * (1.0 + sb * eta);
            N[l] = (1.0 + sa * xi) * (1.0 + sb * eta) * (1.0 + sc * zeta) * 0.125;
        }
        double J[9], Ji[9];
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int b = 0; b < 3; b++) {
                double s = 0.0;
#pragma unroll
                for (int l = 0; l < 8; l++) s += Nd[8 * a + l] * co[3 * l + b];
                J[3 * a + b] = s;
            }
        const double det = inv3(J, Ji);
        double dN[24];
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int l = 0; l < 8; l++)
                dN[8 * a + l] = Ji[3 * a] * Nd[l] + Ji[3 * a + 1] * Nd[8 + l] + Ji[3 * a + 2] * Nd[16 + l];
        const double wd = w * det;
#pragma unroll
        for (int t = 0; t < 10; t++) {
            double gg = dN[li[t]] * dN[lj[t]] + dN[8 + li[t]] * dN[8 + lj[t]] + dN[16 + li[t]] * dN[16 + lj[t]];
            double v = lam * dN[8 * ci[t] + li[t]] * dN[8 * cj[t] + lj[t]] +
                       mu * dN[8 * cj[t] + li[t]] * dN[8 * ci[t] + lj[t]] + (ci[t] == cj[t] ? mu * gg : 0.0);
            acc[t] += wd * v;
        }
#pragma unroll
        for (int t = 0; t < 2; t++) {
            int p = fi[t], q = fj[t];
            double gg = dN[p] * dN[q] + dN[8 + p] * dN[8 + q] + dN[16 + p] * dN[16 + q];
            facc[t] += w * (r2 * gg + N[p] * N[q]) * det;
        }
        if (lane < 8) tacc += w * N[lane] * det;
    }
#pragma unroll
    for (int t = 0; t < 10; t++) {
        int k = lane + 32 * t;
        if (k < 300) {
            size_t o = ((size_t)tile * 300 + k) * 32 + el;
            ke64[o] = acc[t];
            ke32[o] = (float)acc[t];
        }
    }
#pragma unroll
    for (int t = 0; t < 2; t++) {
        int k = lane + 32 * t;
        if (k < 36) kf[((size_t)tile * 36 + k) * 32 + el] = facc[t];
    }
    if (lane < 8) tf[((size_t)tile * 8 + lane) * 32 + el] = tacc;
    if (lane == 0) {
        // 5 tets 6-124, 7-143, 1-657, 4-678, 6-147 (SolveFem.cpp:441-466)
        double a[3], b[3], d[3], p = 0.0;
#define SUBV(o, x, y) for (int q = 0; q < 3; q++) o[q] = co[3 * (x) + q] - co[3 * (y) + q]
        SUBV(a, 5, 0); SUBV(b, 5, 1); SUBV(d, 5, 3);
        p += fabs(1.0 / 6.0 * det3v(a, b, d));
        double s61[3], s64[3];
        for (int q = 0; q < 3; q++) { s61[q] = a[q]; s64[q] = d[q]; }
        SUBV(a, 6, 0); SUBV(b, 6, 3); SUBV(d, 6, 2);
        p += fabs(1.0 / 6.0 * det3v(a, b, d));
        SUBV(a, 0, 5); SUBV(b, 0, 4); SUBV(d, 0, 6);
        p += fabs(1.0 / 6.0 * det3v(a, b, d));
        SUBV(a, 3, 5); SUBV(b, 3, 6); SUBV(d, 3, 7);
        p += fabs(1.0 / 6.0 * det3v(a, b, d));
        SUBV(d, 5, 6);
        p += fabs(1.0 / 6.0 * det3v(s61, s64, d));
#undef SUBV
        vol[e] = p;
    }
}

// tet4: constant-strain Ke (tet4/Tet4Isoparametric.cpp:1-41, detJ =
// sqrt(det(J J')) = |det J|), Helmholtz matrix and T by the 4-point Hammer
// rule (tet4/KeHel.cpp:1-47), volume |det J|/6.  One warp per element.
__global__ void k_tet4_setup(int ne, const int* __restrict__ elem, const double* __restrict__ vertex, double nu,
                             double rmin, double* __restrict__ ke64, float* __restrict__ ke32,
                             double* __restrict__ vol, double* __restrict__ kf, double* __restrict__ tf) {
    const int e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (e >= ne) return;
    const int tile = e >> 5, el = e & 31;
    double co[12];
#pragma unroll
    for (int l = 0; l < 4; l++) {
        int nd = elem[(long)e * 4 + l];
#pragma unroll
        for (int q = 0; q < 3; q++) co[3 * l + q] = vertex[3L * nd + q];
    }
    double J[9], Ji[9];
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) J[3 * a + b] = co[3 * (a + 1) + b] - co[b];
    const double det = inv3(J, Ji);
    const double detJ = sqrt(det * det);
    const double Nd[12] = {-1, 1, 0, 0, -1, 0, 1, 0, -1, 0, 0, 1};
    double dN[12];
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int l = 0; l < 4; l++) dN[4 * a + l] = Ji[3 * a] * Nd[l] + Ji[3 * a + 1] * Nd[4 + l] + Ji[3 * a + 2] * Nd[8 + l];
    const double lam = nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double mu = 1.0 / (2.0 * (1.0 + nu));
    for (int k = lane; k < 78; k += 32) {
        int i, j;
        unpack_ij(k, 12, i, j);
        int ci = i / 4, li = i % 4, cj = j / 4, lj = j % 4;
        double gg = dN[li] * dN[lj] + dN[4 + li] * dN[4 + lj] + dN[8 + li] * dN[8 + lj];
        double v = lam * dN[4 * ci + li] * dN[4 * cj + lj] + mu * dN[4 * cj + li] * dN[4 * ci + lj] + (ci == cj ? mu * gg : 0.0);
        double kv = 1.0 / 6.0 * v * detJ;
        size_t o = ((size_t)tile * 78 + k) * 32 + el;
        ke64[o] = kv;
        ke32[o] = (float)kv;
    }
    const double r = 1.0 / (2.0 * sqrt(3.0)) * rmin;
    const double r2 = r * r;
    const double ga = (5.0 + 3.0 * sqrt(5.0)) / 20.0, gb = (5.0 - sqrt(5.0)) / 20.0;
    if (lane < 10) {
        int p, q;
        unpack_ij(lane, 4, p, q);
        double gg = dN[p] * dN[q] + dN[4 + p] * dN[4 + q] + dN[8 + p] * dN[8 + q];
        double s = 0.0;
        for (int g = 0; g < 4; g++) {
            double sx = g == 0 ? ga : gb, ty = g == 1 ? ga : gb, vz = g == 2 ? ga : gb;
            double N[4] = {1 - sx - ty - vz, sx, ty, vz};
            s += 1.0 / 24.0 * (r2 * gg + N[p] * N[q]) * det;
        }
        kf[((size_t)tile * 10 + lane) * 32 + el] = s;
    } else if (lane < 14) {
        int p = lane - 10;
        double s = 0.0;
        for (int g = 0; g < 4; g++) {
            double sx = g == 0 ? ga : gb, ty = g == 1 ? ga : gb, vz = g == 2 ? ga : gb;
            double N[4] = {1 - sx - ty - vz, sx, ty, vz};
            s += 1.0 / 24.0 * N[p] * det;
        }
        tf[((size_t)tile * 4 + p) * 32 + el] = s;
    } else if (lane == 14) {
        vol[e] = fabs(det3v(J, J + 3, J + 6)) / 6.0;
    }
}

int elem_setup(Ctx& c) {
    size_t nt = c.ntiles;
    TRET(c.ke64.alloc(nt * c.npk * 32));
    TRET(c.ke32.alloc(nt * c.npk * 32));
    TRET(c.kf.alloc(nt * c.nkf * 32));
    TRET(c.tf.alloc(nt * c.nen * 32));
    TRET(c.vol.alloc(c.ne));
    TRET(c.ke64.zero(c.s));
    TRET(c.ke32.zero(c.s));
    TRET(c.kf.zero(c.s));
    TRET(c.tf.zero(c.s));
    int block = 256;
    int grid = (int)(((long)c.ne * 32 + block - 1) / block);
    if (c.nen == 8)
        k_hex8_setup<<<grid, block, 0, c.s>>>(c.ne, c.elem.p, c.vertex.p, c.p.nu, c.p.rmin, c.ke64.p, c.ke32.p, c.vol.p,
                                              c.kf.p, c.tf.p), note_launch();
    else
        k_tet4_setup<<<grid, block, 0, c.s>>>(c.ne, c.elem.p, c.vertex.p, c.p.nu, c.p.rmin, c.ke64.p, c.ke32.p, c.vol.p,
                                              c.kf.p, c.tf.p), note_launch();
    TCK(cudaGetLastError());
    return 0;
}

// ----------------------------------------------------------------- SIMP moduli
__global__ void k_moduli(int ne, int npad, const double* __restrict__ x, double Emin, double Emax, double penal,
                         double* __restrict__ E64, float* __restrict__ E32) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= npad) return;
    double E = 0.0;
    if (e < ne) E = Emin + pow(x[e], penal) * (Emax - Emin);  // SolveFem.cpp:304
    E64[e] = E;
    E32[e] = (float)E;
}

int compute_moduli(Ctx& c, const double* xphys) {
    int npad = c.ntiles * 32;
    if (!c.Ee64.p) { TRET(c.Ee64.alloc(npad)); TRET(c.Ee32.alloc(npad)); }
    k_moduli<<<grid_for(npad, 256, 1 << 20), 256, 0, c.s>>>(c.ne, npad, xphys, c.p.Emin, c.p.Emax, c.p.penal, c.Ee64.p,
                                                           c.Ee32.p), note_launch();
    c.moduli_gen++;
    TCK(cudaGetLastError());
    return 0;
}

// ----------------------------------------------------------------- K(x) u, matrix free
// y[dof] += alpha * E_e * (Ke_e u_e)[dof], Dirichlet columns masked on input
// (u_e entries of fixed DOFs read as 0).  One element per thread; the packed
// symmetric Ke is streamed once from HBM (coalesced AoSoA lines), u is
// gathered through L2/L1 and the 3*NEN outputs are scatter-added with
// red.global.add.  Neighbouring lanes of a lattice-ordered mesh share the
// nodes of a face: the lane-pair combine folds lane i+1's left-face
// contribution into lane i's right-face one when the node ids agree
// (checked, so any mesh stays correct), halving the atomics on such meshes.
//
// STORE (the deterministic form): instead of adding into y, the element's
// 3*NEN outputs go to the scratch y in the AoSoA layout [tile][3 NEN][32],
// and k_node_gather3 adds them node by node in a fixed order.
template <int NEN, class TK, class TU, class TY, bool STORE>
__global__ void __launch_bounds__(128) k_kmv(int ne, const int* __restrict__ conn, const uint32_t* __restrict__ emask,
                                             const TK* __restrict__ ke, const TK* __restrict__ Ee,
                                             const TU* __restrict__ u, TY* __restrict__ y, TK alpha) {
    constexpr int ND = 3 * NEN, NPK = ND * (ND + 1) / 2;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    const int tile = e >> 5, lane = e & 31;
    const bool active = e < ne;
    int nd[NEN];
    TK ue[ND], ye[ND];
    uint32_t msk = 0;
    TK E = 0;
    if (active) {
#pragma unroll
        for (int l = 0; l < NEN; l++) nd[l] = conn[((size_t)tile * NEN + l) * 32 + lane];
        msk = emask[e];
        E = Ee[e] * alpha;
#pragma unroll
        for (int l = 0; l < NEN; l++)
#pragma unroll
            for (int cc = 0; cc < 3; cc++) {
                TU v = u[3L * nd[l] + cc];
                ue[cc * NEN + l] = (msk >> (cc * NEN + l)) & 1u ? TK(0) : TK(v);
            }
        const TK* kp = ke + (size_t)tile * NPK * 32 + lane;
#pragma unroll
        for (int i = 0; i < ND; i++) ye[i] = TK(0);
        int k = 0;
#pragma unroll
        for (int i = 0; i < ND; i++) {
#pragma unroll
            for (int j = i; j < ND; j++, k++) {
                TK a = __ldg(kp + (size_t)k * 32);
                ye[i] += a * ue[j];
                if (j != i) ye[j] += a * ue[i];
            }
        }
    } else {
#pragma unroll
        for (int l = 0; l < NEN; l++) nd[l] = -1;
#pragma unroll
        for (int i = 0; i < ND; i++) ye[i] = TK(0);
    }
#pragma unroll
    for (int i = 0; i < ND; i++) ye[i] *= E;
    if constexpr (STORE) {
        if (active)
#pragma unroll
            for (int i = 0; i < ND; i++) y[((size_t)tile * ND + i) * 32 + lane] = TY(ye[i]);
        return;
    }
    if constexpr (NEN == 8) {
        // lane-pair combine across the shared x-face: my local nodes 1,3,5,7
        // against the next lane's local nodes 0,2,4,6
        bool skip[8] = {false, false, false, false, false, false, false, false};
#pragma unroll
        for (int f = 0; f < 4; f++) {
            const int mine = 2 * f + 1, theirs = 2 * f;
            int nb = __shfl_down_sync(0xffffffffu, nd[theirs], 1);
            bool match = lane < 31 && active && nb == nd[mine] && nb >= 0;
            // the next lane learns that its left-face node was folded into mine
            int up = __shfl_up_sync(0xffffffffu, match ? 1 : 0, 1);
            skip[theirs] = (lane > 0) && up;
#pragma unroll
            for (int cc = 0; cc < 3; cc++) {
                TK o = __shfl_down_sync(0xffffffffu, ye[cc * NEN + theirs], 1);
                if (match) ye[cc * NEN + mine] += o;
            }
        }
        if (active) {
#pragma unroll
            for (int l = 0; l < 8; l++) {
                if (skip[l]) continue;
#pragma unroll
                for (int cc = 0; cc < 3; cc++) atomicAdd(&y[3L * nd[l] + cc], TY(ye[cc * NEN + l]));
            }
        }
    } else {
        if (active) {
#pragma unroll
            for (int l = 0; l < NEN; l++)
#pragma unroll
                for (int cc = 0; cc < 3; cc++) atomicAdd(&y[3L * nd[l] + cc], TY(ye[cc * NEN + l]));
        }
    }
}

// Deterministic scatter, second pass: node n adds, in the fixed order of the
// node-to-element map (entries e * NEN + l, ascending), the contributions its
// elements stored in the first pass: y[3n + c] += sum scr[e][c NEN + l].
template <int NEN, class TY>
__global__ void k_node_gather3(int nn, const int* __restrict__ n2e_ptr, const int* __restrict__ n2e,
                               const TY* __restrict__ scr, TY* __restrict__ y) {
    constexpr int ND = 3 * NEN;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nn) return;
    TY s0 = TY(0), s1 = TY(0), s2 = TY(0);
    const int p1 = n2e_ptr[n + 1];
    for (int p = n2e_ptr[n]; p < p1; p++) {
        const int q = n2e[p], e = q / NEN, l = q - e * NEN;
        const TY* b = scr + ((size_t)(e >> 5) * ND + l) * 32 + (e & 31);
        s0 += b[0];
        s1 += b[NEN * 32];
        s2 += b[2 * NEN * 32];
    }
    y[3L * n] += s0;
    y[3L * n + 1] += s1;
    y[3L * n + 2] += s2;
}
// the same for one value per node (the Helmholtz filter operator)
template <int NEN>
__global__ void k_node_gather1(int nn, const int* __restrict__ n2e_ptr, const int* __restrict__ n2e,
                               const double* __restrict__ scr, double* __restrict__ y) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nn) return;
    double s = 0.0;
    const int p1 = n2e_ptr[n + 1];
    for (int p = n2e_ptr[n]; p < p1; p++) {
        const int q = n2e[p], e = q / NEN, l = q - e * NEN;
        s += scr[((size_t)(e >> 5) * NEN + l) * 32 + (e & 31)];
    }
    y[n] += s;
}

// y = beta*b (or 0 if b == null) before the element scatter
template <class TY>
__global__ void k_init_y(long n, TY* __restrict__ y, const TY* __restrict__ b, TY beta) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        y[i] = b ? beta * b[i] : TY(0);
}
// Dirichlet rows are identity: y[f] = beta*b[f] + alpha*u[f]
template <class TU, class TY>
__global__ void k_fix_rows(int nf, const int* __restrict__ fixed, const TU* __restrict__ u, TY* __restrict__ y,
                           const TY* __restrict__ b, TY alpha, TY beta) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nf) return;
    int f = fixed[i];
    y[f] = (b ? beta * b[f] : TY(0)) + alpha * TY(u[f]);
}

template <class TK, class TU, class TY>
static int launch_kmv(Ctx& c, const TK* ke, const TK* Ee, const TU* u, TY* y, TK alpha) {
    const int block = c.tune.kmv_block, grid = c.ntiles * 32 / block + 1;
    if (c.p.deterministic) {
        // per-element outputs into scratch, then a fixed-order node gather
        TY* scr = reinterpret_cast<TY*>(c.det_scr.p);
        if (!scr) { set_error("deterministic form: no scratch (the option is fixed at creation)"); return TOPO_ERR_ARG; }
        const int gn = (c.nn + 255) / 256;
        if (c.nen == 8) {
            k_kmv<8, TK, TU, TY, true><<<grid, block, 0, c.s>>>(c.ne, c.conn.p, c.emask.p, ke, Ee, u, scr, alpha), note_launch();
            k_node_gather3<8, TY><<<gn, 256, 0, c.s>>>(c.nn, c.n2e_ptr.p, c.n2e.p, scr, y), note_launch();
        } else {
            k_kmv<4, TK, TU, TY, true><<<grid, block, 0, c.s>>>(c.ne, c.conn.p, c.emask.p, ke, Ee, u, scr, alpha), note_launch();
            k_node_gather3<4, TY><<<gn, 256, 0, c.s>>>(c.nn, c.n2e_ptr.p, c.n2e.p, scr, y), note_launch();
        }
        TCK(cudaGetLastError());
        return 0;
    }
    if (c.nen == 8)
        k_kmv<8, TK, TU, TY, false><<<grid, block, 0, c.s>>>(c.ne, c.conn.p, c.emask.p, ke, Ee, u, y, alpha), note_launch();
    else
        k_kmv<4, TK, TU, TY, false><<<grid, block, 0, c.s>>>(c.ne, c.conn.p, c.emask.p, ke, Ee, u, y, alpha), note_launch();
    TCK(cudaGetLastError());
    return 0;
}

// y = K(E) u  (FP64 operator)
int kmatvec(Ctx& c, const double* Ee, const double* u, double* y, int ncase) {
    for (int k = 0; k < ncase; k++) {
        const double* uk = u + (size_t)k * c.ndof;
        double* yk = y + (size_t)k * c.ndof;
        k_init_y<double><<<grid_for(c.ndof, 256), 256, 0, c.s>>>(c.ndof, yk, nullptr, 0.0), note_launch();
        cudaEvent_t e0;
        prof_begin(c, PS_KMV, &e0);
        TRET(launch_kmv<double, double, double>(c, c.ke64.p, Ee, uk, yk, 1.0));
        prof_end(c, PS_KMV, e0);
        if (!c.fixed_h.empty())
            k_fix_rows<double, double><<<grid_for((long)c.fixed_h.size(), 256), 256, 0, c.s>>>(
                (int)c.fixed_h.size(), c.fixed.p, uk, yk, nullptr, 1.0, 0.0), note_launch();
    }
    TCK(cudaGetLastError());
    return 0;
}

// y = K(E) u with an FP32 input vector (the mixed form's preconditioned directions)
int kmatvec_f32in(Ctx& c, const double* Ee, const float* u, double* y) {
    k_init_y<double><<<grid_for(c.ndof, 256), 256, 0, c.s>>>(c.ndof, y, nullptr, 0.0), note_launch();
    cudaEvent_t e0;
    prof_begin(c, PS_KMV, &e0);
    TRET(launch_kmv<double, float, double>(c, c.ke64.p, Ee, u, y, 1.0));
    prof_end(c, PS_KMV, e0);
    if (!c.fixed_h.empty())
        k_fix_rows<float, double><<<grid_for((long)c.fixed_h.size(), 256), 256, 0, c.s>>>(
            (int)c.fixed_h.size(), c.fixed.p, u, y, nullptr, 1.0, 0.0), note_launch();
    TCK(cudaGetLastError());
    return 0;
}

// FP32 element operator for the mixed-precision fine-level smoother:
// y = b - K u (residual form) or y = K u.
int kmatvec32(Ctx& c, const float* u, float* y, const float* b) {
    k_init_y<float><<<grid_for(c.ndof, 256), 256, 0, c.s>>>(c.ndof, y, b, 1.0f), note_launch();
    TRET(launch_kmv<float, float, float>(c, c.ke32.p, c.Ee32.p, u, y, b ? -1.0f : 1.0f));
    if (!c.fixed_h.empty())
        k_fix_rows<float, float><<<grid_for((long)c.fixed_h.size(), 256), 256, 0, c.s>>>(
            (int)c.fixed_h.size(), c.fixed.p, u, y, b, b ? -1.0f : 1.0f, 1.0f), note_launch();
    TCK(cudaGetLastError());
    return 0;
}
int kmatvec64r(Ctx& c, const double* u, double* y, const double* b) {
    k_init_y<double><<<grid_for(c.ndof, 256), 256, 0, c.s>>>(c.ndof, y, b, 1.0), note_launch();
    TRET(launch_kmv<double, double, double>(c, c.ke64.p, c.Ee64.p, u, y, b ? -1.0 : 1.0));
    if (!c.fixed_h.empty())
        k_fix_rows<double, double><<<grid_for((long)c.fixed_h.size(), 256), 256, 0, c.s>>>(
            (int)c.fixed_h.size(), c.fixed.p, u, y, b, b ? -1.0 : 1.0, 1.0), note_launch();
    TCK(cudaGetLastError());
    return 0;
}

// ----------------------------------------------------------------- compliance + sensitivities
// SolveFem.cpp:208-249: per element uKu = u_e' Ke u_e (unmasked u, E = 1 Ke).
// Pass 1 accumulates uKu over the load cases; pass 2 forms fx += E(x) uKu,
// dfdx = -p x^(p-1) (Emax-Emin) uKu, gx += x vol, dgdx = vol / TV with block
// partials (fx, gx) for a deterministic final sum.
template <int NEN>
__global__ void __launch_bounds__(128) k_uku(int ne, long ndof, const int* __restrict__ conn,
                                             const double* __restrict__ ke, const double* __restrict__ U,
                                             double* __restrict__ uku, int accumulate) {
    constexpr int ND = 3 * NEN, NPK = ND * (ND + 1) / 2;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    const int tile = e >> 5, lane = e & 31;
    int nd[NEN];
#pragma unroll
    for (int l = 0; l < NEN; l++) nd[l] = conn[((size_t)tile * NEN + l) * 32 + lane];
    const double* kp = ke + (size_t)tile * NPK * 32 + lane;
    double ue[ND], ye[ND];
#pragma unroll
    for (int l = 0; l < NEN; l++)
#pragma unroll
        for (int cc = 0; cc < 3; cc++) ue[cc * NEN + l] = U[3L * nd[l] + cc];
#pragma unroll
    for (int i = 0; i < ND; i++) ye[i] = 0.0;
    int k = 0;
#pragma unroll
    for (int i = 0; i < ND; i++) {
#pragma unroll
        for (int j = i; j < ND; j++, k++) {
            double a = __ldg(kp + (size_t)k * 32);
            ye[i] += a * ue[j];
            if (j != i) ye[j] += a * ue[i];
        }
    }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < ND; i++) s += ue[i] * ye[i];
    uku[e] = accumulate ? uku[e] + s : s;
}

__global__ void __launch_bounds__(256) k_sens(int ne, const double* __restrict__ uku, const double* __restrict__ x,
                                              const double* __restrict__ vol, double Emin, double Emax, double penal,
                                              double TV, double* __restrict__ dfdx, double* __restrict__ dgdx,
                                              double* __restrict__ part) {
    __shared__ double sm[2 * 32];
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    double v[2] = {0.0, 0.0};
    if (e < ne) {
        const double u = uku[e], xe = x[e];
        v[0] = (Emin + pow(xe, penal) * (Emax - Emin)) * u;
        dfdx[e] = -1.0 * penal * pow(xe, penal - 1) * (Emax - Emin) * u;
        v[1] = xe * vol[e];
        dgdx[e] = vol[e] / TV;
    }
    block_sum<2>(v, sm);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = v[0];
        part[2 * blockIdx.x + 1] = v[1];
    }
}

__global__ void k_sens_final(int nb, const double* __restrict__ part, double TV, double volfrac, int m,
                             double* __restrict__ dsc) {
    __shared__ double sm[2 * 32];
    double v[2] = {0.0, 0.0};
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
        v[0] += part[2 * i];
        v[1] += part[2 * i + 1];
    }
    block_sum<2>(v, sm);
    if (threadIdx.x == 0) {
        dsc[DS_FX] = v[0];
        for (int j = 0; j < m; j++) dsc[DS_GX + j] = 0.0;
        dsc[DS_GX] = v[1] / TV - volfrac;
    }
}

int fem_sensitivities(Ctx& c, const double* xphys, double* dfdx, double* dgdx) {
    int block = 256, nb = (c.ne + block - 1) / block;
    if ((long)c.red.n < 2L * nb) TRET(c.red.alloc(std::max<long>(2L * nb, 4096)));
    if (!c.uku.p) TRET(c.uku.alloc(c.ne));
    // the block solve leaves all cases in one case-interleaved vector: one
    // tensor-core pass gives the uKu sum over the cases
    const bool blk = block_cases(c) && c.blk.u_fresh;
    if (blk) TRET(blk_uku(c, c.blk.U.p, c.uku.p));
    for (int cs = 0; cs < c.ncases && !blk; cs++) {
        const double* Uc = c.U.p + (size_t)cs * c.ndof;
        if (c.nen == 8) k_uku<8><<<(c.ne + 127) / 128, 128, 0, c.s>>>(c.ne, c.ndof, c.conn.p, c.ke64.p, Uc, c.uku.p, cs > 0), note_launch();
        else k_uku<4><<<(c.ne + 127) / 128, 128, 0, c.s>>>(c.ne, c.ndof, c.conn.p, c.ke64.p, Uc, c.uku.p, cs > 0), note_launch();
    }
    k_sens<<<nb, block, 0, c.s>>>(c.ne, c.uku.p, xphys, c.vol.p, c.p.Emin, c.p.Emax, c.p.penal, c.TV, dfdx, dgdx, c.red.p), note_launch();
    k_sens_final<<<1, 1024, 0, c.s>>>(nb, c.red.p, c.TV, c.p.volfrac, c.p.m, c.dsc.p), note_launch();
    // additional constraints (m > 1) get zero sensitivities, like dgdx[j>0]
    // that the reference never writes after VecDuplicateVecs
    if (c.p.m > 1) TCK(cudaMemsetAsync(dgdx + c.ne, 0, sizeof(double) * (size_t)c.ne * (c.p.m - 1), c.s));
    TCK(cudaGetLastError());
    return 0;
}

// ----------------------------------------------------------------- Helmholtz filter operators
// TX = TF x : node n collects T_e[l] x_e of its elements (PDEFilter.cpp:106,147)
template <int NEN>
__global__ void k_tf(int ne, const int* __restrict__ conn, const double* __restrict__ tf, const double* __restrict__ x,
                     double* __restrict__ tx) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    int tile = e >> 5, lane = e & 31;
    double xe = x[e];
#pragma unroll
    for (int l = 0; l < NEN; l++) {
        int nd = conn[((size_t)tile * NEN + l) * 32 + lane];
        atomicAdd(&tx[nd], tf[((size_t)tile * NEN + l) * 32 + lane] * xe);
    }
}
// deterministic form of k_tf: node n sums T_e[l] x_e over its elements in
// the fixed order of the node-to-element map
template <int NEN>
__global__ void k_tf_gather(int nn, const int* __restrict__ n2e_ptr, const int* __restrict__ n2e,
                            const double* __restrict__ tf, const double* __restrict__ x, double* __restrict__ tx) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nn) return;
    double s = 0.0;
    const int p1 = n2e_ptr[n + 1];
    for (int p = n2e_ptr[n]; p < p1; p++) {
        const int q = n2e[p], e = q / NEN, l = q - e * NEN;
        s += tf[((size_t)(e >> 5) * NEN + l) * 32 + (e & 31)] * x[e];
    }
    tx[n] = s;
}
// y = KF r, matrix free over the packed NEN x NEN Helmholtz matrices
// (STORE: the element outputs go to the scratch y as [tile][NEN][32] for
// k_node_gather1, the deterministic form)
template <int NEN, bool STORE>
__global__ void __launch_bounds__(128) k_kf(int ne, const int* __restrict__ conn, const double* __restrict__ kf,
                                            const double* __restrict__ r, double* __restrict__ y) {
    constexpr int NPK = NEN * (NEN + 1) / 2;
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    int tile = e >> 5, lane = e & 31;
    int nd[NEN];
    double re[NEN], ye[NEN];
#pragma unroll
    for (int l = 0; l < NEN; l++) {
        nd[l] = conn[((size_t)tile * NEN + l) * 32 + lane];
        re[l] = r[nd[l]];
        ye[l] = 0.0;
    }
    const double* kp = kf + (size_t)tile * NPK * 32 + lane;
    int k = 0;
#pragma unroll
    for (int i = 0; i < NEN; i++)
#pragma unroll
        for (int j = i; j < NEN; j++, k++) {
            double a = __ldg(kp + (size_t)k * 32);
            ye[i] += a * re[j];
            if (j != i) ye[j] += a * re[i];
        }
    if constexpr (STORE) {
#pragma unroll
        for (int l = 0; l < NEN; l++) y[((size_t)tile * NEN + l) * 32 + lane] = ye[l];
    } else {
#pragma unroll
        for (int l = 0; l < NEN; l++) atomicAdd(&y[nd[l]], ye[l]);
    }
}
// xf_e = sum_l (1/NEN) rx[node_l]  (MatMultTranspose(TFX), PDEFilter.cpp:107,149), optional clamp
template <int NEN>
__global__ void k_tfxT(int ne, const int* __restrict__ conn, const double* __restrict__ rx, double* __restrict__ xf,
                       int clamp, double xmin) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    int tile = e >> 5, lane = e & 31;
    const double w = 1.0 / (double)NEN;
    double s = 0.0;
#pragma unroll
    for (int l = 0; l < NEN; l++) s += w * rx[conn[((size_t)tile * NEN + l) * 32 + lane]];
    if (clamp) {
        if (s < xmin) s = xmin;
        else if (s > 1.0) s = 1.0;
    }
    xf[e] = s;
}

int filter_tf(Ctx& c, const double* x, double* tx) {
    if (c.p.deterministic) {
        const int gn = (c.nn + 255) / 256;
        if (c.nen == 8) k_tf_gather<8><<<gn, 256, 0, c.s>>>(c.nn, c.n2e_ptr.p, c.n2e.p, c.tf.p, x, tx), note_launch();
        else k_tf_gather<4><<<gn, 256, 0, c.s>>>(c.nn, c.n2e_ptr.p, c.n2e.p, c.tf.p, x, tx), note_launch();
        TCK(cudaGetLastError());
        return 0;
    }
    TCK(cudaMemsetAsync(tx, 0, sizeof(double) * c.nn, c.s));
    int g = (c.ne + 127) / 128;
    if (c.nen == 8) k_tf<8><<<g, 128, 0, c.s>>>(c.ne, c.conn.p, c.tf.p, x, tx), note_launch();
    else k_tf<4><<<g, 128, 0, c.s>>>(c.ne, c.conn.p, c.tf.p, x, tx), note_launch();
    TCK(cudaGetLastError());
    return 0;
}
int filter_kf(Ctx& c, const double* r, double* y) {
    TCK(cudaMemsetAsync(y, 0, sizeof(double) * c.nn, c.s));
    int g = (c.ne + 127) / 128;
    cudaEvent_t e0;
    prof_begin(c, PS_FILTER, &e0);
    if (c.p.deterministic) {
        // per-element outputs into scratch, then a fixed-order node gather
        double* scr = c.det_scr.p;
        if (!scr) { set_error("deterministic form: no scratch (the option is fixed at creation)"); return TOPO_ERR_ARG; }
        const int gn = (c.nn + 255) / 256;
        if (c.nen == 8) {
            k_kf<8, true><<<g, 128, 0, c.s>>>(c.ne, c.conn.p, c.kf.p, r, scr), note_launch();
            k_node_gather1<8><<<gn, 256, 0, c.s>>>(c.nn, c.n2e_ptr.p, c.n2e.p, scr, y), note_launch();
        } else {
            k_kf<4, true><<<g, 128, 0, c.s>>>(c.ne, c.conn.p, c.kf.p, r, scr), note_launch();
            k_node_gather1<4><<<gn, 256, 0, c.s>>>(c.nn, c.n2e_ptr.p, c.n2e.p, scr, y), note_launch();
        }
    } else if (c.nen == 8) {
        k_kf<8, false><<<g, 128, 0, c.s>>>(c.ne, c.conn.p, c.kf.p, r, y), note_launch();
    } else {
        k_kf<4, false><<<g, 128, 0, c.s>>>(c.ne, c.conn.p, c.kf.p, r, y), note_launch();
    }
    prof_end(c, PS_FILTER, e0);
    TCK(cudaGetLastError());
    return 0;
}
int filter_tfxT(Ctx& c, const double* rx, double* xf, bool clamp, double xmin) {
    int g = (c.ne + 127) / 128;
    if (c.nen == 8) k_tfxT<8><<<g, 128, 0, c.s>>>(c.ne, c.conn.p, rx, xf, clamp ? 1 : 0, xmin), note_launch();
    else k_tfxT<4><<<g, 128, 0, c.s>>>(c.ne, c.conn.p, rx, xf, clamp ? 1 : 0, xmin), note_launch();
    TCK(cudaGetLastError());
    return 0;
}

// ----------------------------------------------------------------- von Mises (hex8)
// stress/ComputeStress.cpp:53-104: centroid B, sigma = Emax D B u, relaxed by
// sqrt(x), von Mises.  tet4 uses its constant B.
__global__ void k_vm_hex8(int ne, const int* __restrict__ elem, const double* __restrict__ vertex,
                          const double* __restrict__ U, const double* __restrict__ x, double nu, double Emax,
                          double* __restrict__ vm) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    double co[24], ue[24];
    for (int l = 0; l < 8; l++) {
        int nd = elem[(long)e * 8 + l];
        for (int q = 0; q < 3; q++) { co[3 * l + q] = vertex[3L * nd + q]; ue[q * 8 + l] = U[3L * nd + q]; }
    }
    double Nd[24];
    for (int l = 0; l < 8; l++) {
        double sa = (l & 1) ? 1.0 : -1.0, sb = (l & 2) ? 1.0 : -1.0, sc = (l & 4) ? 1.0 : -1.0;
        Nd[l] = 0.125 * sa; Nd[8 + l] = 0.125 * sb; Nd[16 + l] = 0.125 * sc;
    }
    double J[9], Ji[9], dN[24];
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
            double s = 0.0;
            for (int l = 0; l < 8; l++) s += Nd[8 * a + l] * co[3 * l + b];
            J[3 * a + b] = s;
        }
    inv3(J, Ji);
    for (int a = 0; a < 3; a++)
        for (int l = 0; l < 8; l++) dN[8 * a + l] = Ji[3 * a] * Nd[l] + Ji[3 * a + 1] * Nd[8 + l] + Ji[3 * a + 2] * Nd[16 + l];
    double ex = 0, ey = 0, ez = 0, gxy = 0, gyz = 0, gxz = 0;
    for (int l = 0; l < 8; l++) {
        ex += dN[l] * ue[l];
        ey += dN[8 + l] * ue[8 + l];
        ez += dN[16 + l] * ue[16 + l];
        gxy += dN[8 + l] * ue[l] + dN[l] * ue[8 + l];
        gyz += dN[16 + l] * ue[8 + l] + dN[8 + l] * ue[16 + l];
        gxz += dN[16 + l] * ue[l] + dN[l] * ue[16 + l];
    }
    const double lam = nu / ((1.0 + nu) * (1.0 - 2.0 * nu)), mu = 1.0 / (2.0 * (1.0 + nu));
    double tr = ex + ey + ez, sr = sqrt(x[e]);
    double s0 = sr * (Emax * (lam * tr + 2 * mu * ex)), s1 = sr * (Emax * (lam * tr + 2 * mu * ey)),
           s2 = sr * (Emax * (lam * tr + 2 * mu * ez));
    double s3 = sr * (Emax * mu * gxy), s4 = sr * (Emax * mu * gyz), s5 = sr * (Emax * mu * gxz);
    vm[e] = (1.0 / sqrt(2.0)) *
            sqrt((s0 - s1) * (s0 - s1) + (s0 - s2) * (s0 - s2) + (s1 - s2) * (s1 - s2) + 6.0 * (s3 * s3 + s4 * s4 + s5 * s5));
}

int von_mises(Ctx& c, const double* xphys, double* vms) {
    if (c.nen != 8) { set_error("von Mises stress is implemented for hex8 meshes"); return TOPO_ERR_UNSUPPORTED; }
    k_vm_hex8<<<(c.ne + 127) / 128, 128, 0, c.s>>>(c.ne, c.elem.p, c.vertex.p, c.U.p, xphys, c.p.nu, c.p.Emax, vms), note_launch();
    TCK(cudaGetLastError());
    return 0;
}

}  // namespace topo
