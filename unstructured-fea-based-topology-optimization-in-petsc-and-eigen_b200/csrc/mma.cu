// mma.cu -- the Method of Moving Asymptotes on the device (restates
// MMA.cpp of the reference, Aage's TopOpt_in_PETSc MMA).
//
// GenSub is one elementwise pass plus a deterministic reduction for b.  The
// whole dual interior-point solve (SolveDIP with XYZofLAMBDA, DualGrad,
// DualHess, Factorize/Solve, DualLineSearch, DualResidual) runs as ONE
// cooperative kernel: every block sweeps its slice of the design variables,
// block partials meet at a bounded grid barrier, and every block then sums
// all partials in the same order, so all threads hold bit-identical dual
// scalars and take identical control flow without any host round trip.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "ctx.h"

namespace topo {

static std::mutex& coop_mutex() {
    static std::mutex m;
    return m;
}


struct MmaConst {
    double a[kMaxM], c[kMaxM], d[kMaxM];
};

__global__ void k_movelimit(int n, double Xmin, double Xmax, double movlim, const double* __restrict__ x,
                            double* __restrict__ xmin, double* __restrict__ xmax) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double xv = x[i];
    double hi = xv + movlim, lo = xv - movlim;
    xmax[i] = Xmax < hi ? Xmax : hi;  // Min(Xmax, x + movlim)
    xmin[i] = Xmin > lo ? Xmin : lo;  // Max(Xmin, x - movlim)
}

__device__ __forceinline__ double dmax(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double dmin(double a, double b) { return a < b ? a : b; }

// GenSub (MMA.cpp:506-620): asymptotes, bounds, p0/q0/pij/qij, b partials
template <int M>
__global__ void k_gensub(int n, const int* __restrict__ kdev, double asyminit, double asymdec, double asyminc, int robust, int conmod,
                         const double* __restrict__ xv, const double* __restrict__ x1v, const double* __restrict__ x2v,
                         const double* __restrict__ xminv, const double* __restrict__ xmaxv,
                         const double* __restrict__ dfdx, const double* __restrict__ dgdx, double* __restrict__ Lv,
                         double* __restrict__ Uv, double* __restrict__ alf, double* __restrict__ bet,
                         double* __restrict__ p0, double* __restrict__ q0, double* __restrict__ pij,
                         double* __restrict__ qij, double* __restrict__ part) {
    __shared__ double sm[M * 32];
    const int k = *kdev;  // MMA outer iteration, advanced by k_mma_next before this launch
    double bsum[M];
#pragma unroll
    for (int j = 0; j < M; j++) bsum[j] = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double x = xv[i], xmi_ = xminv[i], xma_ = xmaxv[i];
        double L, U;
        if (k < 3) {
            // VecAXPBYPCZ(L, 1, -asyminit, 0, xval, xmax); VecAXPY(L, asyminit, xmin)
            L = 1.0 * x + (-asyminit) * xma_;
            L = L + asyminit * xmi_;
            U = 1.0 * x + asyminit * xma_;
            U = U + (-asyminit) * xmi_;
        } else {
            L = Lv[i];
            U = Uv[i];
            const double x1 = x1v[i], x2 = x2v[i];
            const double helpvar = (x - x1) * (x1 - x2);
            const double gamma = helpvar < 0.0 ? asymdec : (helpvar > 0.0 ? asyminc : 1.0);
            L = x - gamma * (x1 - L);
            U = x + gamma * (U - x1);
            double xmi = dmax(1.0e-5, xma_ - xmi_);
            if (robust == 0) {
                L = dmax(L, x - 10.0 * xmi);
                L = dmin(L, x - 0.01 * xmi);
                U = dmax(U, x + 0.01 * xmi);
                U = dmin(U, x + 10.0 * xmi);
            } else {
                L = dmax(L, x - 100.0 * xmi);
                L = dmin(L, x - 1.0e-4 * xmi);
                U = dmax(U, x + 1.0e-4 * xmi);
                U = dmin(U, x + 100.0 * xmi);
                double xl = xmi_ - 1.0e-5, xh = xma_ + 1.0e-5;
                if (x < xl) { L = x - (xh - x) / 0.9; U = x + (xh - x) / 0.9; }
                if (x > xh) { L = x - (x - xl) / 0.9; U = x + (x - xl) / 0.9; }
            }
        }
        Lv[i] = L;
        Uv[i] = U;
        const double feps = 1.0e-6;
        alf[i] = dmax(xmi_, 0.9 * L + 0.1 * x);
        bet[i] = dmin(xma_, 0.9 * U + 0.1 * x);
        const double df = dfdx[i];
        const double dfp = dmax(0.0, df), dfm = dmax(0.0, -1.0 * df);
        const double ux = U - x, xl = x - L;
        p0[i] = pow(ux, 2.0) * (dfp + 0.001 * fabs(df) + 0.5 * feps / (U - L));
        q0[i] = pow(xl, 2.0) * (dfm + 0.001 * fabs(df) + 0.5 * feps / (U - L));
#pragma unroll
        for (int j = 0; j < M; j++) {
            const double g = dgdx[(long)j * n + i];
            const double gp = dmax(0.0, g), gm = dmax(0.0, -1.0 * g);
            double pv, qv;
            if (conmod) {
                pv = pow(ux, 2.0) * (gp + 0.001 * fabs(g) + 0.5 * feps / (U - L));
                qv = pow(xl, 2.0) * (gm + 0.001 * fabs(g) + 0.5 * feps / (U - L));
            } else {
                pv = pow(ux, 2.0) * gp;
                qv = pow(xl, 2.0) * gm;
            }
            pij[(long)j * n + i] = pv;
            qij[(long)j * n + i] = qv;
            bsum[j] += pv / ux + qv / xl;
        }
    }
    block_sum<M>(bsum, sm);
    if (threadIdx.x == 0)
#pragma unroll
        for (int j = 0; j < M; j++) part[(long)blockIdx.x * M + j] = bsum[j];
}

__global__ void k_gensub_final(int nb, int m, const double* __restrict__ part, const double* __restrict__ gx,
                               double* __restrict__ ms) {
    __shared__ double sm[32];
    for (int j = 0; j < m; j++) {
        double v[1] = {0.0};
        for (int i = threadIdx.x; i < nb; i += blockDim.x) v[0] += part[(long)i * m + j];
        block_sum<1>(v, sm);
        if (threadIdx.x == 0) ms[MS_B + j] = v[0] + (-gx[j]);
        __syncthreads();
    }
}

// ---------------------------------------------------------------- dual interior point
template <int M>
struct DualScalars {
    double lam[M], mu[M], y[M], z;
};

template <int M>
__device__ __forceinline__ void xyz_scalars(DualScalars<M>& s, const MmaConst& k) {
    // XYZofLAMBDA scalar part (MMA.cpp:693-701), a0 = 1
    double lamai = 0.0;
#pragma unroll
    for (int i = 0; i < M; i++) {
        if (s.lam[i] < 0.0) s.lam[i] = 0;
        s.y[i] = dmax(0.0, s.lam[i] - k.c[i]);
        lamai += s.lam[i] * k.a[i];
    }
    s.z = dmax(0.0, 10.0 * (lamai - 1.0));
}

// sums all blocks' partials (identical order on every block)
template <int NV>
__device__ __forceinline__ void gather_partials(const double* part, int nb, double (&out)[NV], double* sm) {
    double v[NV];
#pragma unroll
    for (int q = 0; q < NV; q++) v[q] = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x)
#pragma unroll
        for (int q = 0; q < NV; q++) v[q] += __ldcg(part + (long)b * NV + q);
    block_sum<NV>(v, sm);
    __shared__ double bc[NV];
    if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < NV; q++) bc[q] = v[q];
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NV; q++) out[q] = bc[q];
    __syncthreads();
}

template <int M>
__global__ void __launch_bounds__(256) k_solvedip(int n, double* __restrict__ xout, const double* __restrict__ p0,
                                                  const double* __restrict__ q0, const double* __restrict__ pij,
                                                  const double* __restrict__ qij, const double* __restrict__ Lv,
                                                  const double* __restrict__ Uv, const double* __restrict__ alf,
                                                  const double* __restrict__ bet, double* __restrict__ ms,
                                                  MmaConst kc, double tol, double* __restrict__ part1,
                                                  double* __restrict__ part2, GridBarrier bar) {
    constexpr int NV1 = M + M * M;
    __shared__ double sm[NV1 * 32];
    double b[M];
#pragma unroll
    for (int j = 0; j < M; j++) b[j] = ms[MS_B + j];
    DualScalars<M> s;
#pragma unroll
    for (int j = 0; j < M; j++) { s.lam[j] = kc.c[j] / 2.0; s.mu[j] = 1.0; }
    double epsi = 1.0, err = 1.0;
    int total = 0;
    bool ok = true;
    const int tid0 = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    while (epsi > tol && ok) {
        int loop = 0;
        while (err > 0.9 * epsi && loop < 100) {
            loop++;
            total++;
            // XYZofLAMBDA + DualGrad + DualHess sums (same x(lambda))
            xyz_scalars<M>(s, kc);
            double acc[NV1];
#pragma unroll
            for (int q = 0; q < NV1; q++) acc[q] = 0.0;
            for (int i = tid0; i < n; i += stride) {
                double pj = p0[i], qj = q0[i], pv[M], qv[M];
#pragma unroll
                for (int j = 0; j < M; j++) {
                    pv[j] = pij[(long)j * n + i];
                    qv[j] = qij[(long)j * n + i];
                    pj += pv[j] * s.lam[j];
                    qj += qv[j] * s.lam[j];
                }
                const double L = Lv[i], U = Uv[i];
                const double sp = sqrt(pj), sq = sqrt(qj);
                const double xp = (sp * L + sq * U) / (sp + sq);
                double x = xp;
                if (x < alf[i]) x = alf[i];
                if (x > bet[i]) x = bet[i];
                xout[i] = x;
                const double ux = U - x, xl = x - L;
                double df2 = -1.0 / (2.0 * pj / pow(ux, 3.0) + 2.0 * qj / pow(xl, 3.0));
                if (xp < alf[i]) df2 = 0.0;
                if (xp > bet[i]) df2 = 0.0;
                double PQ[M];
#pragma unroll
                for (int j = 0; j < M; j++) {
                    acc[j] += pv[j] / ux + qv[j] / xl;
                    PQ[j] = pv[j] / pow(ux, 2.0) - qv[j] / pow(xl, 2.0);
                }
#pragma unroll
                for (int a = 0; a < M; a++)
#pragma unroll
                    for (int c2 = 0; c2 < M; c2++) acc[M + a * M + c2] += (PQ[a] * df2) * PQ[c2];
            }
            block_sum<NV1>(acc, sm);
            if (threadIdx.x == 0)
#pragma unroll
                for (int q = 0; q < NV1; q++) part1[(long)blockIdx.x * NV1 + q] = acc[q];
            if (!grid_sync(bar)) { ok = false; break; }
            double tot[NV1];
            gather_partials<NV1>(part1, gridDim.x, tot, sm);
            // DualGrad (MMA.cpp:756-758), then grad = -grad - epsi/lam (:657-659)
            double grad[M], H[M * M];
#pragma unroll
            for (int j = 0; j < M; j++) {
                grad[j] = tot[j] + (-b[j] - kc.a[j] * s.z - s.y[j]);
                grad[j] = -1.0 * grad[j] - epsi / s.lam[j];
            }
            // DualHess tail (MMA.cpp:826-854)
#pragma unroll
            for (int q = 0; q < M * M; q++) H[q] = tot[M + q];
            double lamai = 0.0;
#pragma unroll
            for (int j = 0; j < M; j++) {
                if (s.lam[j] < 0.0) s.lam[j] = 0.0;
                lamai += s.lam[j] * kc.a[j];
                if (s.lam[j] > kc.c[j]) H[j * M + j] += -1.0;
                H[j * M + j] += -s.mu[j] / s.lam[j];
            }
            if (lamai > 0.0)
#pragma unroll
                for (int j = 0; j < M; j++)
#pragma unroll
                    for (int q = 0; q < M; q++) H[j * M + q] += -10.0 * kc.a[j] * kc.a[q];
            double tr = 0.0;
#pragma unroll
            for (int i = 0; i < M; i++) tr += H[i * M + i];
            double corr = 1e-4 * tr / M;
            if (-1.0 * corr < 1.0e-7) corr = -1.0e-7;
#pragma unroll
            for (int i = 0; i < M; i++) H[i * M + i] += corr;
            // Factorize + Solve: LU without pivoting (MMA.cpp:936-969)
#pragma unroll
            for (int ss = 0; ss < M - 1; ss++)
#pragma unroll
                for (int i = ss + 1; i < M; i++) {
                    H[i * M + ss] = H[i * M + ss] / H[ss * M + ss];
#pragma unroll
                    for (int j = ss + 1; j < M; j++) H[i * M + j] = H[i * M + j] - H[i * M + ss] * H[ss * M + j];
                }
#pragma unroll
            for (int i = 1; i < M; i++) {
                double a = 0.0;
#pragma unroll
                for (int j = 0; j < i; j++) a = a - H[i * M + j] * grad[j];
                grad[i] = grad[i] + a;
            }
            grad[M - 1] = grad[M - 1] / H[(M - 1) * M + (M - 1)];
#pragma unroll
            for (int i = M - 2; i >= 0; i--) {
                double a = grad[i];
#pragma unroll
                for (int j = i + 1; j < M; j++) a = a - H[i * M + j] * grad[j];
                grad[i] = a / H[i * M + i];
            }
            double sv[2 * M];
#pragma unroll
            for (int j = 0; j < M; j++) sv[j] = grad[j];
#pragma unroll
            for (int i = 0; i < M; i++) sv[M + i] = -s.mu[i] + epsi / s.lam[i] - sv[i] * s.mu[i] / s.lam[i];
            // DualLineSearch (MMA.cpp:870-888)
            double theta = 1.005;
#pragma unroll
            for (int i = 0; i < M; i++) {
                if (theta < -1.01 * sv[i] / s.lam[i]) theta = -1.01 * sv[i] / s.lam[i];
                if (theta < -1.01 * sv[i + M] / s.mu[i]) theta = -1.01 * sv[i + M] / s.mu[i];
            }
            theta = 1.0 / theta;
#pragma unroll
            for (int i = 0; i < M; i++) {
                s.lam[i] = s.lam[i] + theta * sv[i];
                s.mu[i] = s.mu[i] + theta * sv[i + M];
            }
            // XYZofLAMBDA + DualResidual sums
            xyz_scalars<M>(s, kc);
            double rs[M];
#pragma unroll
            for (int j = 0; j < M; j++) rs[j] = 0.0;
            for (int i = tid0; i < n; i += stride) {
                double pj = p0[i], qj = q0[i], pv[M], qv[M];
#pragma unroll
                for (int j = 0; j < M; j++) {
                    pv[j] = pij[(long)j * n + i];
                    qv[j] = qij[(long)j * n + i];
                    pj += pv[j] * s.lam[j];
                    qj += qv[j] * s.lam[j];
                }
                const double L = Lv[i], U = Uv[i];
                const double sp = sqrt(pj), sq = sqrt(qj);
                double x = (sp * L + sq * U) / (sp + sq);
                if (x < alf[i]) x = alf[i];
                if (x > bet[i]) x = bet[i];
                xout[i] = x;
#pragma unroll
                for (int j = 0; j < M; j++) rs[j] += pv[j] / (U - x) + qv[j] / (x - L);
            }
            block_sum<M>(rs, sm);
            if (threadIdx.x == 0)
#pragma unroll
                for (int q = 0; q < M; q++) part2[(long)blockIdx.x * M + q] = rs[q];
            if (!grid_sync(bar)) { ok = false; break; }
            double rt[M];
            gather_partials<M>(part2, gridDim.x, rt, sm);
            double nrI = 0.0;
#pragma unroll
            for (int j = 0; j < M; j++) {
                double r1 = rt[j] + (-b[j] - kc.a[j] * s.z - s.y[j] + s.mu[j]);
                double r2 = 0.0 + (s.mu[j] * s.lam[j] - epsi);
                if (nrI < fabs(r1)) nrI = fabs(r1);
                if (nrI < fabs(r2)) nrI = fabs(r2);
            }
            err = nrI;
        }
        epsi = epsi * 0.1;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
#pragma unroll
        for (int j = 0; j < M; j++) { ms[MS_LAM + j] = s.lam[j]; ms[MS_MU + j] = s.mu[j]; ms[MS_Y + j] = s.y[j]; }
        ms[MS_Z] = s.z;
        ms[MS_ITS] = (double)total;
        ms[MS_ERR] = err;
    }
}

// DesignChange (MMA.cpp:391-410): max |x - xold|, xold = x
__global__ void k_design_change(int n, const double* __restrict__ x, double* __restrict__ xold,
                                double* __restrict__ part) {
    __shared__ double sm[32];
    double ch = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double d = fabs(x[i] - xold[i]);
        ch = ch > d ? ch : d;
        xold[i] = x[i];
    }
    ch = block_max(ch, sm);
    if (threadIdx.x == 0) part[blockIdx.x] = ch;
}
__global__ void k_max_final(int nb, const double* __restrict__ part, double* __restrict__ out) {
    __shared__ double sm[32];
    double v = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) v = v > part[i] ? v : part[i];
    v = block_max(v, sm);
    if (threadIdx.x == 0) *out = v;
}

// KKTresidual (MMA.cpp:412-480) sums: [norm2^2 partial, normInf partial]
template <int M>
__global__ void k_kkt(int n, const double* __restrict__ x, const double* __restrict__ xmin,
                      const double* __restrict__ xmax, const double* __restrict__ df0, const double* __restrict__ dg,
                      const double* __restrict__ ms, double* __restrict__ part) {
    __shared__ double sm[32];
    double n2[1] = {0.0}, ni = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double ri = df0[i];
#pragma unroll
        for (int j = 0; j < M; j++) ri += ms[MS_LAM + j] * dg[(long)j * n + i];
        double mu_min = 0.0, mu_max = 0.0;
        if (x[i] < xmin[i] + 1.0e-5 && ri > 0.0) mu_min = ri;
        if (x[i] > xmax[i] - 1.0e-5 && ri < 0.0) mu_max = -ri;
        ri += -mu_min + mu_max;
        n2[0] += pow(ri, 2.0);
        ni = dmax(fabs(ri), ni);
        double resi = mu_min * (x[i] - xmin[i]);
        n2[0] += pow(resi, 2.0);
        ni = dmax(fabs(resi), ni);
        resi = mu_max * (xmax[i] - x[i]);
        n2[0] += pow(resi, 2.0);
        ni = dmax(fabs(resi), ni);
    }
    block_sum<1>(n2, sm);
    double mx = block_max(ni, sm);
    if (threadIdx.x == 0) { part[2L * blockIdx.x] = n2[0]; part[2L * blockIdx.x + 1] = mx; }
}
__global__ void k_kkt_final(int nb, const double* __restrict__ part, double* __restrict__ out) {
    __shared__ double sm[32];
    double v[1] = {0.0}, mx = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) { v[0] += part[2L * i]; mx = dmax(mx, part[2L * i + 1]); }
    block_sum<1>(v, sm);
    mx = block_max(mx, sm);
    if (threadIdx.x == 0) { out[0] = v[0]; out[1] = mx; }
}

// k++ of MMA::GenSub (MMA.cpp:508), on the device so that a replayed graph advances it
__global__ void k_mma_next(int* __restrict__ k) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *k += 1;
}

// ---------------------------------------------------------------- host side
constexpr int kMmaBlocks = 296;

int mma_alloc(Ctx& c) {
    if (c.L.p) return 0;
    const int n = c.ne, m = c.p.m;
    TRET(c.L.alloc(n)); TRET(c.Uas.alloc(n)); TRET(c.alpha.alloc(n)); TRET(c.beta.alloc(n));
    TRET(c.p0.alloc(n)); TRET(c.q0.alloc(n));
    TRET(c.pij.alloc((size_t)n * m)); TRET(c.qij.alloc((size_t)n * m));
    TRET(c.xo1.alloc(n)); TRET(c.xo2.alloc(n));
    TRET(c.xo1.zero(c.s)); TRET(c.xo2.zero(c.s)); TRET(c.L.zero(c.s)); TRET(c.Uas.zero(c.s));
    TRET(c.mma_scal.alloc(kMmaSlots + 2L * 2048 * (kMaxM + kMaxM * kMaxM)));
    TRET(c.mma_scal.zero(c.s));
    TRET(c.bar.alloc(2));
    TRET(c.bar.zero(c.s));
    TRET(c.bar_err.alloc(1));
    TRET(c.bar_err.zero(c.s));
    c.a.assign(m, 0.0);
    c.c.assign(m, 1000.0);
    c.d.assign(m, 0.0);
    return 0;
}

int mma_movelimit(Ctx& c, double Xmin, double Xmax, double movlim, const double* x, double* xmin, double* xmax) {
    k_movelimit<<<(c.ne + 255) / 256, 256, 0, c.s>>>(c.ne, Xmin, Xmax, movlim, x, xmin, xmax), note_launch();
    TCK(cudaGetLastError());
    return 0;
}

template <int M>
static int update_m(Ctx& c, double* x, const double* dfdx, const double* gx_dev, const double* dgdx,
                    const double* xmin, const double* xmax) {
    const int n = c.ne;
    double* ms = c.mma_scal.p;
    double* part = ms + kMmaSlots;
    int* kdev = c.di.p + DI_MMA_K;
    k_mma_next<<<1, 32, 0, c.s>>>(kdev), note_launch();
    k_gensub<M><<<kMmaBlocks, 256, 0, c.s>>>(n, kdev, c.asyminit, c.asymdec, c.asyminc, c.robust_type,
                                            c.constraint_mod, x, c.xo1.p, c.xo2.p, xmin, xmax, dfdx, dgdx, c.L.p,
                                            c.Uas.p, c.alpha.p, c.beta.p, c.p0.p, c.q0.p, c.pij.p, c.qij.p, part), note_launch();
    k_gensub_final<<<1, 256, 0, c.s>>>(kMmaBlocks, M, part, gx_dev, ms), note_launch();
    TCK(cudaGetLastError());
    // Update: xo2 <- xo1, xo1 <- xval (MMA.cpp:496-497)
    TCK(cudaMemcpyAsync(c.xo2.p, c.xo1.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, c.s));
    TCK(cudaMemcpyAsync(c.xo1.p, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, c.s));
    // SolveDIP as one cooperative launch
    int dev, dev_sms = 0;
    TCK(cudaGetDevice(&dev));
    TCK(cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, dev));
    int occ = 0;
    TCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_solvedip<M>, 256, 0));
    // Co-residency: the grid barrier needs every block of the grid resident at
    // once.  A direct launch (one at a time per process, under coop_mutex)
    // leaves one block slot per SM free, and the launches from replayed step
    // graphs that can run at once take at most one block per SM together
    // (stepgraph.cu: a context's own part-1 graphs run one at a time per device
    // and process, chained on an event; inside a batch graph every instance's
    // grid is capped at its share, coop_blocks), so the direct and the graph
    // grids can run side by side without any waiting on blocks that cannot
    // start.
    const int cap = c.sg.dd ? (c.sg.coop_blocks > 0 ? std::min(c.sg.coop_blocks, dev_sms) : dev_sms)
                            : dev_sms * std::max(occ - 1, 1);
    int blocks = std::max(1, std::min(cap, std::min(2048, (n + 255) / 256)));
    MmaConst kc{};
    for (int j = 0; j < M; j++) { kc.a[j] = c.a[j]; kc.c[j] = c.c[j]; kc.d[j] = c.d[j]; }
    double tol = 1.0e-9 * std::sqrt((double)(M + n));
    double* part1 = part;
    double* part2 = part + (size_t)2048 * (M + M * M);
    TCK(cudaMemsetAsync(c.bar.p, 0, 2 * sizeof(unsigned), c.s));
    TCK(cudaMemsetAsync(c.bar_err.p, 0, sizeof(int), c.s));
    GridBarrier gb{c.bar.p, c.bar.p + 1, c.bar_err.p, c.wait.barrier_spins, c.wait.hold};
    const double* p0 = c.p0.p; const double* q0 = c.q0.p; const double* pij = c.pij.p; const double* qij = c.qij.p;
    const double* Lp = c.L.p; const double* Up = c.Uas.p; const double* al = c.alpha.p; const double* be = c.beta.p;
    int nn = n;
    void* args[] = {&nn, &x, &p0, &q0, &pij, &qij, &Lp, &Up, &al, &be, &ms, &kc, &tol, &part1, &part2, &gb};
    if (c.sg.dd) {
        // device-driven step: a cooperative kernel node in the step graph; the
        // iteration count and the barrier flag are read once the step is done
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(blocks);
        cfg.blockDim = dim3(256);
        cfg.stream = c.s;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeCooperative;
        at[0].val.cooperative = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        TCK(cudaLaunchKernelExC(&cfg, (const void*)k_solvedip<M>, args));
        note_launch();
        return 0;
    }
    int* herr = reinterpret_cast<int*>(c.hsc.h + 201);
    *herr = 0;
    {
        // one cooperative grid in flight per process: concurrent jobs (serving)
        // never hold parts of the device against each other's grid barriers
        std::lock_guard<std::mutex> lk(coop_mutex());
        TCK(cudaLaunchCooperativeKernel((void*)k_solvedip<M>, dim3(blocks), dim3(256), args, 0, c.s));
        note_launch();
        TCK(cudaMemcpyAsync(c.hsc.h + 200, ms + MS_ITS, sizeof(double), cudaMemcpyDeviceToHost, c.s));
        TCK(cudaMemcpyAsync(herr, c.bar_err.p, sizeof(int), cudaMemcpyDeviceToHost, c.s));
        TCK(cudaStreamSynchronize(c.s));
    }
    c.info.mma_inner_its = (int)c.hsc.h[200];
    if (*herr) { set_error("MMA dual solve: grid barrier timed out"); return TOPO_ERR_TIMEOUT; }
    return 0;
}

int mma_update(Ctx& c, double* x, const double* dfdx, const double* gx_dev, const double* dgdx, const double* xmin,
               const double* xmax) {
    TRET(mma_alloc(c));
    switch (c.p.m) {
        case 1: return update_m<1>(c, x, dfdx, gx_dev, dgdx, xmin, xmax);
        case 2: return update_m<2>(c, x, dfdx, gx_dev, dgdx, xmin, xmax);
        case 3: return update_m<3>(c, x, dfdx, gx_dev, dgdx, xmin, xmax);
        case 4: return update_m<4>(c, x, dfdx, gx_dev, dgdx, xmin, xmax);
        default: set_error("MMA supports 1 <= m <= %d constraints", kMaxM); return TOPO_ERR_UNSUPPORTED;
    }
}

int mma_design_change(Ctx& c, const double* x, double* xold, double* ch_dev) {
    TRET(mma_alloc(c));
    double* part = c.mma_scal.p + kMmaSlots;
    k_design_change<<<kMmaBlocks, 256, 0, c.s>>>(c.ne, x, xold, part), note_launch();
    k_max_final<<<1, 256, 0, c.s>>>(kMmaBlocks, part, ch_dev), note_launch();
    TCK(cudaGetLastError());
    return 0;
}

int mma_kkt(Ctx& c, const double* x, const double* dfdx, const double* gx_dev, const double* dgdx, const double* xmin,
            const double* xmax, double* n2, double* ninf) {
    TRET(mma_alloc(c));
    double* part = c.mma_scal.p + kMmaSlots;
    double* out = c.dsc.p + DS_KKT;
    switch (c.p.m) {
        case 1: k_kkt<1><<<kMmaBlocks, 256, 0, c.s>>>(c.ne, x, xmin, xmax, dfdx, dgdx, c.mma_scal.p, part), note_launch(); break;
        case 2: k_kkt<2><<<kMmaBlocks, 256, 0, c.s>>>(c.ne, x, xmin, xmax, dfdx, dgdx, c.mma_scal.p, part), note_launch(); break;
        case 3: k_kkt<3><<<kMmaBlocks, 256, 0, c.s>>>(c.ne, x, xmin, xmax, dfdx, dgdx, c.mma_scal.p, part), note_launch(); break;
        default: k_kkt<4><<<kMmaBlocks, 256, 0, c.s>>>(c.ne, x, xmin, xmax, dfdx, dgdx, c.mma_scal.p, part), note_launch(); break;
    }
    k_kkt_final<<<1, 256, 0, c.s>>>(kMmaBlocks, part, out), note_launch();
    TCK(cudaGetLastError());
    double h[2 + 3 * kMaxM + 1], gxh[kMaxM];
    TCK(cudaMemcpyAsync(c.hsc.h + 210, out, 2 * sizeof(double), cudaMemcpyDeviceToHost, c.s));
    TCK(cudaMemcpyAsync(c.hsc.h + 212, c.mma_scal.p, 13 * sizeof(double), cudaMemcpyDeviceToHost, c.s));
    TCK(cudaMemcpyAsync(c.hsc.h + 230, gx_dev, c.p.m * sizeof(double), cudaMemcpyDeviceToHost, c.s));
    TCK(cudaStreamSynchronize(c.s));
    (void)h;
    (void)gxh;
    double nrm2 = c.hsc.h[210], nri = c.hsc.h[211];
    const double* ms = c.hsc.h + 212;
    double ri = 0.0;
    for (int j = 0; j < c.p.m; j++) ri += ms[MS_LAM + j] * (c.a[j] * ms[MS_Z] + ms[MS_Y + j] - c.hsc.h[230 + j]);
    nrm2 += ri * ri;
    nri = std::max(std::fabs(ri), nri);
    *n2 = std::sqrt(nrm2);
    *ninf = nri;
    return 0;
}

}  // namespace topo
