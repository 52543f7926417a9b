// common.cuh -- shared device/host helpers for the sm_100a topology-optimisation
// library: error plumbing, device buffers, deterministic block reductions and a
// bounded grid barrier for cooperative (persistent) kernels.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstring>
#include <cstdio>
#include <string>
#include <utility>
#include <vector>

#include "../../include/topo.h"

namespace topo {

// ----------------------------------------------------------------- errors
void set_error(const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* file, int line);

#define TCK(...)                                                         \
    do {                                                                 \
        cudaError_t e_ = (__VA_ARGS__);                                  \
        if (e_ != cudaSuccess) return ::topo::cuda_fail(e_, __FILE__, __LINE__); \
    } while (0)
#define TRET(...)                     \
    do {                              \
        int r_ = (__VA_ARGS__);       \
        if (r_ < 0) return r_;        \
    } while (0)

// ----------------------------------------------------------------- launch accounting
// Process-wide count of kernel launches issued by this library (every launch
// site is followed by note_launch()); read through topo_kernel_launches().
long& launch_counter();
inline void note_launch() { __atomic_fetch_add(&launch_counter(), 1L, __ATOMIC_RELAXED); }

// ----------------------------------------------------------------- programmatic dependent launch
// A kernel launched by launch_k(pdl = true, ...) may be scheduled while the
// previous kernel in the stream is still running, once that kernel has
// executed pdl_trigger() in all its CTAs.  It must call pdl_wait() -- which
// returns when every prerequisite grid has completed and its writes are
// visible -- before it reads or writes anything a kernel still running could
// touch; before the wait it may only read data written ahead of the solve
// (matrix values and patterns, diagonal inverses).  Both are no-ops for a
// kernel launched without the attribute.
#ifdef __CUDACC__
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
#endif

template <typename... KArgs, typename... Args>
inline cudaError_t launch_k(bool pdl, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                            Args&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    note_launch();
    return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

// ----------------------------------------------------------------- buffers
// Owning device allocation (cudaMalloc); never copied, only moved.
template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    DBuf& operator=(DBuf&& o) noexcept {
        if (this != &o) { reset(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
        return *this;
    }
    ~DBuf() { reset(); }
    void reset() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    int alloc(size_t count) {
        reset();
        if (count == 0) count = 1;
        cudaError_t e = cudaMalloc(&p, count * sizeof(T));
        if (e != cudaSuccess) {
            p = nullptr;
            cudaGetLastError();
            set_error("cudaMalloc of %zu bytes failed: %s", count * sizeof(T), cudaGetErrorString(e));
            return TOPO_ERR_OOM;
        }
        n = count;
        return 0;
    }
    int upload(const T* h, size_t count, cudaStream_t s) {
        TRET(alloc(count));
        if (count) TCK(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
        return 0;
    }
    int upload(const std::vector<T>& v, cudaStream_t s) { return upload(v.data(), v.size(), s); }
    int zero(cudaStream_t s) {
        if (p) TCK(cudaMemsetAsync(p, 0, n * sizeof(T), s));
        return 0;
    }
    size_t bytes() const { return n * sizeof(T); }
};

// pinned host scratch for small device->host readbacks
struct PinnedScalars {
    double* h = nullptr;
    size_t n = 0;
    int alloc(size_t count) {
        if (h) cudaFreeHost(h);
        h = nullptr;
        cudaError_t e = cudaMallocHost(&h, count * sizeof(double));
        if (e != cudaSuccess) { cudaGetLastError(); h = nullptr; set_error("cudaMallocHost failed"); return TOPO_ERR_OOM; }
        n = count;
        return 0;
    }
    ~PinnedScalars() { if (h) cudaFreeHost(h); }
};

#ifdef __CUDACC__
// ----------------------------------------------------------------- device helpers
constexpr int kWarp = 32;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Warp reduce-scatter of NV per-lane sums (NV a power of two, at most 32):
// each halving step sends one half of the remaining sums to the partner lane
// and keeps the other half, NV - 1 shuffles in all instead of 5 per sum; the
// lanes that still share a sum then add it with a butterfly.  On return lane
// l holds the warp's total of sum l % NV.  The order of additions is fixed.
template <int NV>
__device__ __forceinline__ double warp_reduce_scatter(double (&a)[NV]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int h = NV / 2; h >= 1; h >>= 1) {
        const bool up = lane & h;
#pragma unroll
        for (int k = 0; k < h; k++) {
            const double send = up ? a[k] : a[k + h];
            const double keep = up ? a[k + h] : a[k];
            a[k] = keep + __shfl_xor_sync(0xffffffffu, send, h);
        }
    }
    double r = a[0];
#pragma unroll
    for (int o = NV; o < 32; o <<= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
    return r;
}

// Deterministic block reduction of NV sums; result valid in thread 0.
// smem must hold NV * 32 doubles.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* smem) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] = warp_sum(v[k]);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; k++) smem[k * 32 + wid] = v[k];
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) {
            double t = lane < nw ? smem[k * 32 + lane] : 0.0;
            v[k] = warp_sum(t);
        }
    }
    __syncthreads();
}

__device__ __forceinline__ double block_max(double v, double* smem) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    v = warp_max(v);
    __syncthreads();
    if (lane == 0) smem[wid] = v;
    __syncthreads();
    if (wid == 0) {
        double t = lane < nw ? smem[lane] : 0.0;
        v = warp_max(t);
    }
    __syncthreads();
    return v;
}

// Bounded grid barrier for kernels launched with cudaLaunchCooperativeKernel
// (co-residency guaranteed by the launch).  Every wait polls at most
// spin_limit times (kBarrierSpin by default, about a second); on expiry it
// raises *err and returns false so the kernel can unwind instead of hanging
// the device.  hold != 0 is the test form of a barrier that never opens:
// the last block to arrive does not release the others, so every block's
// wait runs out and the kernel reports the timeout.
constexpr unsigned kBarrierSpin = 1u << 24;

struct GridBarrier {
    unsigned* count;   // arrivals in the current generation
    unsigned* gen;     // generation counter
    int* err;          // set to 1 on timeout
    unsigned spin_limit;
    int hold;
};

__device__ __forceinline__ bool grid_sync(const GridBarrier& b) {
    __syncthreads();
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        s_ok = 1;
        volatile unsigned* vgen = b.gen;
        unsigned g = *vgen;
        __threadfence();
        unsigned arrived = atomicAdd(b.count, 1u) + 1u;
        if (arrived == gridDim.x && !b.hold) {
            *b.count = 0;
            __threadfence();
            atomicAdd(b.gen, 1u);
        } else {
            unsigned spins = 0;
            while (*vgen == g) {
                if (++spins > b.spin_limit || *(volatile int*)b.err) {
                    atomicExch(b.err, 1);
                    s_ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return s_ok != 0;
}

// ----------------------------------------------------------------- level-0 sliced ELLPACK values
// One slot of a 32-row slice holds 9 values per row (a 3x3 block) in 288
// elements: the first G*VPL entries of all 32 rows as 16-byte vectors
// (VPL = 16/sizeof(T) entries per row and vector, G vectors), then the
// remaining entries row-interleaved.  A warp reads a slot with G 16-byte
// loads and 9 - G*VPL scalar loads per lane (float: 2 + 1, double: 4 + 1,
// half: 1 + 1) instead of 9 scalar loads.
template <class T>
__host__ __device__ __forceinline__ size_t sell_idx(size_t slot, int e, int lane) {
    constexpr int VPL = 16 / (int)sizeof(T), G = 9 / VPL;
    const size_t base = slot * 288;
    if (e < G * VPL) return base + (size_t)(e / VPL) * 32 * VPL + (size_t)lane * VPL + (e % VPL);
    return base + (size_t)G * 32 * VPL + (size_t)(e - G * VPL) * 32 + lane;
}
template <class T, class TV>
__device__ __forceinline__ void sell_load9(const T* __restrict__ S, size_t slot, int lane, TV (&av)[9]) {
    constexpr int VPL = 16 / (int)sizeof(T), G = 9 / VPL;
    const T* p = S + slot * 288;
    T raw[9];
#pragma unroll
    for (int g = 0; g < G; g++) {
        const uint4 t = __ldg(reinterpret_cast<const uint4*>(p + g * 32 * VPL + lane * VPL));
        memcpy(raw + g * VPL, &t, 16);
    }
#pragma unroll
    for (int r = 0; r < 9 - G * VPL; r++) raw[G * VPL + r] = p[G * 32 * VPL + r * 32 + lane];
#pragma unroll
    for (int e = 0; e < 9; e++) av[e] = (TV)raw[e];
}

#endif  // __CUDACC__

inline int grid_for(long n, int block, int max_blocks = 148 * 64) {
    long g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > max_blocks) g = max_blocks;
    return (int)g;
}

}  // namespace topo
