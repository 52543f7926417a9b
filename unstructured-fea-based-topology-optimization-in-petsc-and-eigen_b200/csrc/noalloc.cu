// noalloc.cu -- compliance and sensitivities of a given displacement without
// any device allocation.
//
// Some callers cannot call cudaMalloc at the time they need this reduction:
// code running inside a stream-ordered pipeline that must not synchronise the
// device (cudaMalloc/cudaFree can), hosts whose allocations all go through a
// pool they do not own, and embedded or real-time drivers that forbid
// allocation after start-up.  They pass every input and output; the only
// scratch (one pair of per-block partial sums per thread block and a
// completion counter) lives in the file-scope array below, which every GPU
// that loads this library holds until the process exits.
//
// Limits and sharing: at most kNoallocMaxBlocks blocks of kNoallocBlock
// elements (n_elems <= 1,048,576); larger meshes are rejected.  All calls
// share the one array and it keeps the last call's contents: the counter is
// cleared at the start of every call, and two calls whose work overlaps on
// the GPU (different streams, no ordering between them) race on it.
#include <cuda_runtime.h>

#include <mutex>

#include "ctx.h"

namespace topo {

constexpr int kNoallocBlock = 128;
constexpr int kNoallocMaxBlocks = 8192;
constexpr long kNoallocMaxElems = (long)kNoallocBlock * kNoallocMaxBlocks;

// [0, 2*kNoallocMaxBlocks): per-block (fx, gx) partials; [2*kNoallocMaxBlocks]:
// completion counter (as unsigned int in the first word)
static __device__ __align__(256) double g_noalloc_scratch[2 * kNoallocMaxBlocks + 32];

// SolveFem.cpp:208-249 on a plain layout: element e's Ke (E = 1) is the
// packed upper triangle (row-major, i <= j) at ke[e*npk ...]; element e's
// nodes at element[e*nen ...]; u is 3*n_nodes with DOF 3n+c.  One warp per
// element: lanes own packed entries, the warp sums u'Ke u.  The last block to
// finish adds all partials in block order (deterministic) and writes
// out[0] = fx, out[1] = gx = sum x vol / TV - volfrac.
template <int NEN>
__global__ void __launch_bounds__(kNoallocBlock) k_sens_noalloc(int ne, const int* __restrict__ element,
                                                                const double* __restrict__ ke,
                                                                const double* __restrict__ x,
                                                                const double* __restrict__ vol,
                                                                const double* __restrict__ u, double Emin,
                                                                double Emax, double penal, double TV, double volfrac,
                                                                double* __restrict__ dfdx, double* __restrict__ dgdx,
                                                                double* __restrict__ out, double* __restrict__ scratch) {
    constexpr int ND = 3 * NEN, NPK = ND * (ND + 1) / 2;
    __shared__ double sm[2 * 32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    constexpr int kWarps = kNoallocBlock / 32;
    double v[2] = {0.0, 0.0};
    // each warp walks kNoallocBlock / kWarps = 32 elements of this block's range
    for (int q = 0; q < kNoallocBlock / kWarps; q++) {
        const int e = blockIdx.x * kNoallocBlock + wib * (kNoallocBlock / kWarps) + q;
        if (e >= ne) break;
        double ue_lane = 0.0;  // lane l < ND holds u of local DOF l = c*NEN + node
        if (lane < ND) {
            const int c = lane / NEN, l = lane % NEN;
            ue_lane = u[3L * element[(long)e * NEN + l] + c];
        }
        const double* kp = ke + (size_t)e * NPK;
        // every lane runs every chunk (uniform trip count) so the shuffles of
        // u stay converged; lanes past the packed entries contribute zero
        double s = 0.0;
        for (int kb = 0; kb < NPK; kb += 32) {
            const int k = kb + lane;
            int i = 0, j = 0;
            double a = 0.0;
            if (k < NPK) {
                int rem = k, len = ND;
                while (rem >= len) { rem -= len; i++; len--; }
                j = i + rem;
                a = kp[k];
            }
            const double ui = __shfl_sync(0xffffffffu, ue_lane, i);
            const double uj = __shfl_sync(0xffffffffu, ue_lane, j);
            if (k < NPK) s += (i == j ? 1.0 : 2.0) * a * ui * uj;
        }
        s = warp_sum(s);
        if (lane == 0) {
            const double xe = x[e];
            v[0] += (Emin + pow(xe, penal) * (Emax - Emin)) * s;
            dfdx[e] = -1.0 * penal * pow(xe, penal - 1) * (Emax - Emin) * s;
            v[1] += xe * vol[e];
            dgdx[e] = vol[e] / TV;
        }
    }
    block_sum<2>(v, sm);
    unsigned* counter = reinterpret_cast<unsigned*>(scratch + 2 * kNoallocMaxBlocks);
    if (threadIdx.x == 0) {
        scratch[2 * blockIdx.x] = v[0];
        scratch[2 * blockIdx.x + 1] = v[1];
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double t[2] = {0.0, 0.0};
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
        t[0] += __ldcg(scratch + 2 * b);
        t[1] += __ldcg(scratch + 2 * b + 1);
    }
    block_sum<2>(t, sm);
    if (threadIdx.x == 0) {
        out[0] = t[0];
        out[1] = t[1] / TV - volfrac;
    }
}

// device address of the scratch array, looked up once per device
static double* scratch_ptr(int* rc) {
    static std::mutex mu;
    static double* ptrs[64] = {nullptr};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        *rc = cuda_fail(e == cudaSuccess ? cudaErrorInvalidDevice : e, __FILE__, __LINE__);
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(mu);
    if (!ptrs[dev]) {
        double* p = nullptr;
        e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_noalloc_scratch);
        if (e != cudaSuccess) {
            cudaGetLastError();
            *rc = cuda_fail(e, __FILE__, __LINE__);
            return nullptr;
        }
        ptrs[dev] = p;
    }
    *rc = 0;
    return ptrs[dev];
}

}  // namespace topo

using namespace topo;

extern "C" int topo_fem_sensitivities_noalloc(int nen, int n_elems, const int32_t* element_d, const double* ke_d,
                                              const double* xphys_d, const double* vol_d, const double* u_d,
                                              double Emin, double Emax, double penal, double total_volume,
                                              double volfrac, double* dfdx_d, double* dgdx_d, double* fx_gx_d,
                                              void* stream) {
    if (nen != 8 && nen != 4) { set_error("nen must be 8 (hex8) or 4 (tet4)"); return TOPO_ERR_ARG; }
    if (n_elems < 1 || !element_d || !ke_d || !xphys_d || !vol_d || !u_d || !dfdx_d || !dgdx_d || !fx_gx_d) {
        set_error("null argument or empty mesh");
        return TOPO_ERR_ARG;
    }
    if ((long)n_elems > kNoallocMaxElems) {
        set_error("topo_fem_sensitivities_noalloc handles at most %ld elements (got %d): its scratch is a fixed "
                  "device array; use topo_fem_obj_sens for larger meshes",
                  kNoallocMaxElems, n_elems);
        return TOPO_ERR_ARG;
    }
    if (!(total_volume > 0.0)) { set_error("total volume must be positive"); return TOPO_ERR_ARG; }
    int rc = 0;
    double* scratch = scratch_ptr(&rc);
    if (!scratch) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    // the completion counter must start at zero on every call
    TCK(cudaMemsetAsync(scratch + 2 * kNoallocMaxBlocks, 0, sizeof(double), s));
    const int blocks = (n_elems + kNoallocBlock - 1) / kNoallocBlock;
    if (nen == 8)
        k_sens_noalloc<8><<<blocks, kNoallocBlock, 0, s>>>(n_elems, element_d, ke_d, xphys_d, vol_d, u_d, Emin, Emax,
                                                           penal, total_volume, volfrac, dfdx_d, dgdx_d, fx_gx_d,
                                                           scratch), note_launch();
    else
        k_sens_noalloc<4><<<blocks, kNoallocBlock, 0, s>>>(n_elems, element_d, ke_d, xphys_d, vol_d, u_d, Emin, Emax,
                                                           penal, total_volume, volfrac, dfdx_d, dgdx_d, fx_gx_d,
                                                           scratch), note_launch();
    TCK(cudaGetLastError());
    return 0;
}
