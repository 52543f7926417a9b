// block.cu -- the k-load block operator K(x) [u_1 .. u_k] for load cases that
// share one stiffness matrix (compliance and its sensitivity summed over the
// cases; the per-case quantities are those of SolveFem.cpp:208-249).
//
// Block vectors are case-interleaved: entry (dof, case) at dof*KB + case with
// KB in {4, 8, 16} (cases >= ncases are zero), so the KB values of one DOF
// are one contiguous 32/64/128-byte run.
//
// Per element the product Y_e = E_e Ke_e U_e (24x24 by 24xKB for hex8) is a
// dense contraction and runs on the FP64 tensor cores (mma.m8n8k4.f64; the
// tcgen05 instruction family has no FP64 kind).  One warp owns one element at
// a time: its packed Ke (300 doubles) is brought into shared memory by the
// TMA engine (cp.async.bulk, completion on a per-warp mbarrier, a ring of
// ST copies in flight per warp, 2 or 3 picked by the autotuner: 2 leaves room
// for more CTAs per SM), the U_e fragments are gathered from
// global memory one phase ahead, and the outputs accumulate in a
// shared-memory image of the chunk's nodes.  Elements are grouped (host
// side, once per mesh) into chunks of <= 32 spatially close elements (Morton
// order of the centroids) and each chunk into phases of <= kWarps elements
// that share no node, so a phase's warps update the shared image without
// atomics; a chunk's image is added to global memory once, which cuts the
// global atomics about 3x against per-element scatter.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "ctx.h"

namespace topo {

constexpr int kWarps = 4;      // warps (= elements per phase) per CTA
constexpr int kChunkElems = 32;

// ----------------------------------------------------------------- host: chunks and phases
// spread the low 21 bits of v to every third bit (3D Morton code)
static uint64_t spread21(uint64_t v) {
    v &= 0x1FFFFFull;
    v = (v | (v << 32)) & 0x1F00000000FFFFull;
    v = (v | (v << 16)) & 0x1F0000FF0000FFull;
    v = (v | (v << 8)) & 0x100F00F00F00F00Full;
    v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

int blk_build_schedule(Ctx& c, int node_cap) {
    BlockState& B = c.blk;
    const int nen = c.nen, ne = c.ne;
    if (c.nn >= (1 << 29)) { set_error("block operator: at most 2^29 nodes"); return TOPO_ERR_UNSUPPORTED; }
    // Morton order of the element centroids on a grid of the mean element
    // size h = (node bounding box volume / elements)^(1/3); on a lattice the
    // rounded centroid is the element's lattice index, so 32 consecutive
    // codes are an aligned 4x4x2 brick, which the phase colouring below
    // splits into 8 node-disjoint phases of 4 (one element per warp of a
    // 4-warp CTA; small CTAs keep 5 per SM resident, so 40 element-matrix
    // copies per SM are in flight with 2 per warp)
    double lo[3] = {1e300, 1e300, 1e300}, nlo[3] = {1e300, 1e300, 1e300}, nhi[3] = {-1e300, -1e300, -1e300};
    for (int i = 0; i < c.nn; i++)
        for (int d = 0; d < 3; d++) {
            nlo[d] = std::min(nlo[d], c.vertex_h[3L * i + d]);
            nhi[d] = std::max(nhi[d], c.vertex_h[3L * i + d]);
        }
    std::vector<double> cen((size_t)ne * 3);
    for (int e = 0; e < ne; e++)
        for (int d = 0; d < 3; d++) {
            double s = 0.0;
            for (int l = 0; l < nen; l++) s += c.vertex_h[3L * c.elem_h[(long)e * nen + l] + d];
            s /= nen;
            cen[3L * e + d] = s;
            lo[d] = std::min(lo[d], s);
        }
    double vol = 1.0;
    for (int d = 0; d < 3; d++) vol *= std::max(nhi[d] - nlo[d], 1e-300);
    const double h = std::max(std::cbrt(vol / std::max(ne, 1)), 1e-300);
    std::vector<std::pair<uint64_t, int>> key(ne);
    for (int e = 0; e < ne; e++) {
        uint64_t q[3];
        for (int d = 0; d < 3; d++)
            q[d] = (uint64_t)std::min(2097151.0, std::max(0.0, std::nearbyint((cen[3L * e + d] - lo[d]) / h)));
        key[e] = {spread21(q[0]) | (spread21(q[1]) << 1) | (spread21(q[2]) << 2), e};
    }
    std::sort(key.begin(), key.end());

    // greedy chunks: <= kChunkElems elements and <= node_cap distinct nodes
    std::vector<int> stamp(c.nn, -1);
    std::vector<int> ch_begin;  // into key order
    int nch = 0, nodes_in = 0, elems_in = 0;
    for (int q = 0; q < ne; q++) {
        const int e = key[q].second;
        int fresh = 0;
        for (int l = 0; l < nen; l++) fresh += (nch == 0 || stamp[c.elem_h[(long)e * nen + l]] != nch - 1) ? 1 : 0;
        if (nch == 0 || elems_in == kChunkElems || nodes_in + fresh > node_cap) {
            ch_begin.push_back(q);
            nch++;
            nodes_in = elems_in = 0;
            fresh = 0;
            for (int l = 0; l < nen; l++) {
                const int nd = c.elem_h[(long)e * nen + l];
                if (stamp[nd] != nch - 1) { stamp[nd] = nch - 1; fresh++; }
            }
        } else {
            for (int l = 0; l < nen; l++) stamp[c.elem_h[(long)e * nen + l]] = nch - 1;
        }
        nodes_in += fresh;
        elems_in++;
    }
    ch_begin.push_back(ne);

    // per chunk: sorted local node list, then phases of <= kWarps elements
    // with no shared node (first fit over a per-node phase bitmask)
    std::vector<int> ch_ph(1, 0), ph_sl(1, 0), ch_np(1, 0), ch_nodes;
    std::vector<int> sl_elem, sl_gn;
    std::vector<uint16_t> sl_lc;
    std::vector<uint32_t> sl_mask;
    sl_elem.reserve(ne);
    std::vector<uint64_t> used(c.nn, 0);
    std::vector<int> local(c.nn, -1);
    int max_nodes = 0, max_ph = 0;
    for (int k = 0; k < nch; k++) {
        const int q0 = ch_begin[k], q1 = ch_begin[k + 1];
        std::vector<int> nodes;
        for (int q = q0; q < q1; q++)
            for (int l = 0; l < nen; l++) nodes.push_back(c.elem_h[(long)key[q].second * nen + l]);
        std::sort(nodes.begin(), nodes.end());
        nodes.erase(std::unique(nodes.begin(), nodes.end()), nodes.end());
        for (size_t i = 0; i < nodes.size(); i++) local[nodes[i]] = (int)i;
        max_nodes = std::max(max_nodes, (int)nodes.size());
        std::vector<std::vector<int>> phases;
        for (int q = q0; q < q1; q++) {
            const int e = key[q].second;
            uint64_t u = 0;
            for (int l = 0; l < nen; l++) u |= used[c.elem_h[(long)e * nen + l]];
            int p = 0;
            while (p < 64 && (((u >> p) & 1ull) || (p < (int)phases.size() && (int)phases[p].size() >= kWarps))) p++;
            if (p >= 64) { set_error("block schedule: more than 64 phases in a chunk"); return TOPO_ERR_UNSUPPORTED; }
            if (p == (int)phases.size()) phases.emplace_back();
            phases[p].push_back(e);
            for (int l = 0; l < nen; l++) used[c.elem_h[(long)e * nen + l]] |= 1ull << p;
        }
        for (auto& ph : phases) {
            for (int e : ph) {
                sl_elem.push_back(e);
                uint32_t m = 0;
                for (int l = 0; l < nen; l++) {
                    const int nd = c.elem_h[(long)e * nen + l];
                    sl_gn.push_back(nd);
                    sl_lc.push_back((uint16_t)local[nd]);
                    for (int cc = 0; cc < 3; cc++)
                        if (c.dof_fixed_h[3L * nd + cc]) m |= 1u << (cc * nen + l);
                }
                sl_mask.push_back(m);
            }
            ph_sl.push_back((int)sl_elem.size());
        }
        max_ph = std::max(max_ph, (int)phases.size());
        ch_ph.push_back((int)ph_sl.size() - 1);
        for (int nd : nodes) {
            // bits 29..31: Dirichlet flags of the node's x, y, z DOFs
            int enc = nd;
            for (int cc = 0; cc < 3; cc++)
                if (c.dof_fixed_h[3L * nd + cc]) enc |= 1 << (29 + cc);
            ch_nodes.push_back(enc);
            used[nd] = 0;
            local[nd] = -1;
        }
        ch_np.push_back((int)ch_nodes.size());
    }
    B.nchunks = nch;
    B.nphases = (int)ph_sl.size() - 1;
    B.max_nodes = max_nodes;
    B.max_phases = max_ph;
    B.node_cap = node_cap;
    cudaStream_t s = c.s;
    TRET(B.ch_ph.upload(ch_ph, s));
    TRET(B.ph_sl.upload(ph_sl, s));
    TRET(B.ch_np.upload(ch_np, s));
    TRET(B.ch_nodes.upload(ch_nodes, s));
    TRET(B.sl_elem.upload(sl_elem, s));
    TRET(B.sl_gn.upload(sl_gn, s));
    TRET(B.sl_lc.upload(sl_lc, s));
    TRET(B.sl_mask.upload(sl_mask, s));
    return 0;
}

__host__ __device__ __forceinline__ int pk_idx(int i, int j, int n) {
    if (i > j) { int t = i; i = j; j = t; }
    return i * n - (i * (i - 1)) / 2 + (j - i);
}

// Bank layout of the block operator's packed element matrices.  Lane l of a
// warp reads the A-fragment entry (8 mt + l/4, 4 kt + l%4) of the packed
// symmetric Ke; a 64-bit shared load is served per half-warp, without bank
// conflicts when its 16 lanes' distinct entries sit at positions distinct
// mod 16.  The packed entries are therefore stored permuted: entry k at
// perm[k], with perm built from a colouring of the entries by position mod
// 16 in which every half-warp fragment gets distinct colours (a greedy
// colouring with a fixed seed; the identity if none is found).
int blk_bank_perm(int nd, std::vector<int>& perm) {
    const int npk = nd * (nd + 1) / 2, MT = (nd + 7) / 8, KT = (nd + 3) / 4;
    std::vector<std::vector<int>> groups;
    for (int mt = 0; mt < MT; mt++)
        for (int kt = 0; kt < KT; kt++)
            for (int h = 0; h < 2; h++) {
                std::vector<int> g;
                for (int l = 16 * h; l < 16 * h + 16; l++) {
                    const int i = 8 * mt + l / 4, j = 4 * kt + l % 4;
                    if (i < nd && j < nd) g.push_back(pk_idx(i, j, nd));
                }
                std::sort(g.begin(), g.end());
                g.erase(std::unique(g.begin(), g.end()), g.end());
                groups.push_back(g);
            }
    std::vector<std::vector<int>> member(npk);
    std::vector<int> weight(npk, 0);
    for (int gi = 0; gi < (int)groups.size(); gi++)
        for (int k : groups[gi]) {
            member[k].push_back(gi);
            weight[k] += (int)groups[gi].size();
        }
    uint64_t rs = 0x2545F4914F6CDD1Dull;
    auto rnd = [&]() {
        rs ^= rs << 13;
        rs ^= rs >> 7;
        rs ^= rs << 17;
        return rs;
    };
    perm.resize(npk);
    for (int t = 0; t < 200; t++) {
        std::vector<int> order(npk);
        for (int k = 0; k < npk; k++) order[k] = k;
        for (int k = npk - 1; k > 0; k--) std::swap(order[k], order[(int)(rnd() % (uint64_t)(k + 1))]);
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return weight[a] > weight[b]; });
        int left[16];
        for (int r = 0; r < 16; r++) left[r] = (npk - r + 15) / 16;
        std::vector<int> col(npk, -1);
        std::vector<uint32_t> used(groups.size(), 0u);
        bool ok = true;
        for (int k : order) {
            uint32_t bad = 0;
            for (int g : member[k]) bad |= used[g];
            int best = -1;
            uint64_t bkey = 0;
            for (int r = 0; r < 16; r++) {
                if (((bad >> r) & 1u) || left[r] == 0) continue;
                const uint64_t key = ((uint64_t)left[r] << 32) | (rnd() & 0xffffffffull);
                if (best < 0 || key > bkey) { best = r; bkey = key; }
            }
            if (best < 0) { ok = false; break; }
            col[k] = best;
            left[best]--;
            for (int g : member[k]) used[g] |= 1u << best;
        }
        if (!ok) continue;
        int next[16];
        for (int r = 0; r < 16; r++) next[r] = r;
        for (int k = 0; k < npk; k++) {
            perm[k] = next[col[k]];
            next[col[k]] += 16;
        }
        return 1;
    }
    for (int k = 0; k < npk; k++) perm[k] = k;
    return 0;
}

// keb[slot][perm[k]] = Ke entry k of element sl_elem[slot] (from the AoSoA tiles)
__global__ void k_keb_gather(int nslot, int npk, const int* __restrict__ sl_elem, const int* __restrict__ perm,
                             const double* __restrict__ ke, double* __restrict__ keb) {
    const int slot = blockIdx.x;
    if (slot >= nslot) return;
    const int e = sl_elem[slot], t = e >> 5, lane = e & 31;
    for (int k = threadIdx.x; k < npk; k += blockDim.x)
        keb[(size_t)slot * npk + perm[k]] = ke[((size_t)t * npk + k) * 32 + lane];
}

// Es[slot] = E[sl_elem[slot]] (refreshed when the moduli change)
__global__ void k_es_gather(int nslot, const int* __restrict__ sl_elem, const double* __restrict__ E,
                            double* __restrict__ Es) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nslot) Es[i] = E[sl_elem[i]];
}

// ----------------------------------------------------------------- device: TMA bulk copy + mbarrier
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait: false after `limit` clock cycles (Ctx::WaitLimits, about a
// second by default)
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, unsigned long long limit) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > limit) return false;
    return true;
}
// global -> shared bulk copy through the TMA engine (no multicast)
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// D(8x8) += A(8x4, row) B(4x8, col), FP64 tensor cores.  Lane l holds
// A[l/4][l%4], B[l%4][l/4] and D[l/4][2(l%4) + {0,1}].
__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}


struct BlkArgs {
    int nchunks;
    const int* ch_ph;        // chunk -> phase range
    const int* ph_sl;        // phase -> slot range
    const int* ch_np;        // chunk -> node-list range
    const int* ch_nodes;     // chunk-local node -> global node | Dirichlet flags << 29
    const int* sl_elem;      // slot -> element
    const int* sl_gn;        // slot -> nen global nodes
    const uint16_t* sl_lc;   // slot -> nen chunk-local nodes
    const uint32_t* sl_mask; // slot -> fixed local DOFs (bit c*nen + l)
    const double* keb;       // slot -> packed Ke, entry k at kperm[k]
    const int* kperm;
    const double* Es;        // slot -> element modulus
    int max_nodes;           // largest chunk node count (shared image rows)
    int* err;
    unsigned long long wait_cycles;  // bound of each copy wait
    int hold;                // test form: issue no copy, so every wait runs out
};

// MODE 0: y[dof][case] += alpha E_e (Ke_e U_e) over all elements, Dirichlet
//         columns masked on input, Dirichlet rows not written (the caller
//         sets them).
// MODE 1: uku[e] = sum_case u_e' Ke_e u_e (E = 1, unmasked u).
template <int NEN, int KB, int MODE, class TU, int ST>
__global__ void __launch_bounds__(kWarps * 32, 5) k_blk_kmv(BlkArgs a, const TU* __restrict__ u, double* __restrict__ y,
                                                       double alpha, double* __restrict__ uku) {
    constexpr int ND = 3 * NEN, NPK = ND * (ND + 1) / 2;
    constexpr int MT = (ND + 7) / 8, KT = (ND + 3) / 4, NT = (KB + 7) / 8;
    constexpr int NVL = 3 * KB;  // values per node in the shared image
    extern __shared__ __align__(128) unsigned char smraw[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smraw);                        // [kWarps][ST]
    double* kes = reinterpret_cast<double*>(smraw + 128 * ((kWarps * ST * 8 + 127) / 128));
    double* yl = kes + kWarps * ST * NPK;                                  // [max_nodes][3][KB]
    __shared__ int s_abort;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nch = a.nchunks;
    if (threadIdx.x == 0) s_abort = 0;
    if (lane == 0)
        for (int s = 0; s < ST; s++) mbar_init(&bar[warp * ST + s], 1);
    fence_mbar_init();
    // per-lane A-fragment offsets into the packed Ke
    int aoff[MT][KT];
#pragma unroll
    for (int mt = 0; mt < MT; mt++)
#pragma unroll
        for (int kt = 0; kt < KT; kt++) {
            const int i = 8 * mt + (lane >> 2), j = 4 * kt + (lane & 3);
            aoff[mt][kt] = (i < ND && j < ND) ? a.kperm[pk_idx(i, j, ND)] : -1;
        }
    if (MODE == 0)
        for (int i = threadIdx.x; i < a.max_nodes * NVL; i += blockDim.x) yl[i] = 0.0;
    __syncthreads();

    // producer (issue) and consumer cursors over this CTA's phases
    int pc = blockIdx.x, pp = pc < nch ? a.ch_ph[pc] : 0, pq = 0;
    int cc = blockIdx.x, cp = cc < nch ? a.ch_ph[cc] : 0, cq = 0;
    uint32_t parity = 0, pending = 0;
    auto issue = [&]() {
        const int s0 = a.ph_sl[pp], cnt = a.ph_sl[pp + 1] - s0;
        const int st = pq % ST;
        if (warp < cnt && !a.hold) {
            if (lane == 0) {
                fence_proxy_async();
                mbar_expect_tx(&bar[warp * ST + st], NPK * 8);
                bulk_g2s(kes + (warp * ST + st) * NPK, a.keb + (size_t)(s0 + warp) * NPK, NPK * 8,
                         &bar[warp * ST + st]);
            }
            pending |= 1u << st;
        }
        pq++;
        if (++pp == a.ch_ph[pc + 1]) {
            pc += gridDim.x;
            pp = pc < nch ? a.ch_ph[pc] : 0;
        }
    };
    for (int i = 0; i < ST - 1 && pc < nch; i++) issue();

    // Per-element data of the elements this warp owns in the next phases,
    // fetched ahead so that no dependent global load sits on the critical
    // path: the slot record (global and chunk-local node ids, Dirichlet mask,
    // modulus) two phases ahead, the U_e fragments (B operand: DOF
    // 4kt + lane%4, case lane/4 + 8nt) one phase ahead.
    // Lane-level view of one element's fragments (fixed by the mma layout):
    // - B row d = 4 kt + lane%4 is DOF (comp, node) with node = d % NEN and
    //   comp = d / NEN: for hex8 node 4 (kt & 1) + lane%4 and comp kt / 2,
    //   for tet4 node lane%4 and comp kt, so a lane's six B rows touch NBN
    //   element nodes (2 or 1);
    // - D row 8 mt + lane/4 is node lane/4 (hex8; comp mt) or (lane/4) % 4
    //   (tet4; comp 2 mt + lane/16), one element node per lane.
    // The per-element record a lane loads is therefore NBN global node ids,
    // one D-row node id, the Dirichlet mask and the modulus.
    constexpr int NBN = NEN == 8 ? 2 : 1;
    const int lD = NEN == 8 ? (lane >> 2) : ((lane >> 2) & 3);
    struct Meta {
        int gb[NBN];    // global nodes of this lane's B rows
        int dn;         // MODE 0: chunk-local node of this lane's D rows; MODE 1: global node
        uint32_t msk;
        int e;
        double E;
        bool has;
    };
    auto load_meta = [&](int ch, int ph, Meta& m) {
        m.has = false;
        if (ch >= nch) return;
        const int s0 = a.ph_sl[ph];
        if (warp >= a.ph_sl[ph + 1] - s0) return;
        const int slot = s0 + warp;
        m.has = true;
        const int* gns = a.sl_gn + (size_t)slot * NEN;
#pragma unroll
        for (int h = 0; h < NBN; h++) m.gb[h] = gns[4 * h + (lane & 3)];
        m.dn = MODE == 0 ? (int)a.sl_lc[(size_t)slot * NEN + lD] : gns[lD];
        m.msk = MODE == 0 ? a.sl_mask[slot] : 0u;
        if (MODE == 1) m.e = a.sl_elem[slot];
        m.E = MODE == 0 ? a.Es[slot] : 1.0;
    };
    auto load_b = [&](const Meta& m, double (&bf)[KT][NT]) {
        if (!m.has) return;
        const uint32_t lm = m.msk >> (lane & 3);  // bit 4 kt: B row d = 4 kt + lane%4 is fixed
        long base[NBN];
#pragma unroll
        for (int h = 0; h < NBN; h++) base[h] = (long)m.gb[h] * (3 * KB) + (lane >> 2);
#pragma unroll
        for (int kt = 0; kt < KT; kt++) {
            const int h = NEN == 8 ? (kt & 1) : 0;
            const int comp = NEN == 8 ? (kt >> 1) : kt;
            const bool fixed = (lm >> (4 * kt)) & 1u;
#pragma unroll
            for (int nt = 0; nt < NT; nt++) {
                const int n = (lane >> 2) + 8 * nt;
                bf[kt][nt] = (n < KB && !fixed) ? (double)u[base[h] + comp * KB + 8 * nt] : 0.0;
            }
        }
    };
    auto next_phase = [&](int& ch, int& ph) {
        if (ch >= nch) return;
        if (++ph == a.ch_ph[ch + 1]) {
            ch += gridDim.x;
            ph = ch < nch ? a.ch_ph[ch] : 0;
        }
    };
    Meta mc, mn, mnn;
    double bcur[KT][NT], bnxt[KT][NT];
#pragma unroll
    for (int kt = 0; kt < KT; kt++)
#pragma unroll
        for (int nt = 0; nt < NT; nt++) bcur[kt][nt] = bnxt[kt][nt] = 0.0;
    int c1 = cc, p1 = cp;
    next_phase(c1, p1);
    int c2 = c1, p2 = p1;
    next_phase(c2, p2);
    load_meta(cc, cp, mc);
    load_b(mc, bcur);
    load_meta(c1, p1, mn);

    bool ok = true;
    while (cc < nch) {
        if (pc < nch) issue();
        const int st = cq % ST;
        load_meta(c2, p2, mnn);
        load_b(mn, bnxt);
        if (mc.has) {
            if (mbar_wait(&bar[warp * ST + st], (parity >> st) & 1u, a.wait_cycles)) {
                parity ^= 1u << st;
                pending &= ~(1u << st);
            } else {
                ok = false;
                if (lane == 0) { s_abort = 1; atomicExch(a.err, 1); }
            }
            const double* ks = kes + (warp * ST + st) * NPK;
            const double sc = MODE == 0 ? alpha * mc.E : 1.0;
            double q = 0.0;
#pragma unroll
            for (int nt = 0; nt < NT; nt++) {
                // MT independent accumulation chains, interleaved over k
                double acc[MT][2];
#pragma unroll
                for (int mt = 0; mt < MT; mt++) acc[mt][0] = acc[mt][1] = 0.0;
                if (ok) {
#pragma unroll
                    for (int kt = 0; kt < KT; kt++)
#pragma unroll
                        for (int mt = 0; mt < MT; mt++) {
                            // hex8: 24 = 3 x 8 rows and 6 x 4 columns, every index valid
                            const double av = (ND % 8 == 0 || aoff[mt][kt] >= 0) ? ks[aoff[mt][kt]] : 0.0;
                            dmma(acc[mt], av, bcur[kt][nt]);
                        }
                }
                const int n0 = 2 * (lane & 3) + 8 * nt;
                // this lane's D rows: one element node, component comp(mt)
                const long dbase = MODE == 0 ? (long)mc.dn * NVL + n0 : (long)mc.dn * (3 * KB) + n0;
#pragma unroll
                for (int mt = 0; mt < MT; mt++) {
                    const int dof = 8 * mt + (lane >> 2);
                    if (dof < ND) {
                        const int comp = NEN == 8 ? mt : 2 * mt + (lane >> 4);
                        if (MODE == 0) {
                            // the lane's two cases are one aligned 16-byte pair: n0 is even, the
                            // node and component offsets are multiples of KB >= 4 doubles, and
                            // the image starts 8 * ST * NPK doubles (a multiple of 16 bytes)
                            // after the 128-byte aligned element-matrix ring
                            if (n0 < KB) {
                                double2* yp = reinterpret_cast<double2*>(yl + dbase + comp * KB);
                                double2 cur = *yp;
                                cur.x += sc * acc[mt][0];
                                cur.y += sc * acc[mt][1];
                                *yp = cur;
                            }
                        } else {
#pragma unroll
                            for (int i = 0; i < 2; i++)
                                if (n0 + i < KB) q += acc[mt][i] * (double)u[dbase + comp * KB + i];
                        }
                    }
                }
            }
            if (MODE == 1) {
                q = warp_sum(q);
                if (lane == 0) uku[mc.e] = q;
            }
        }
        __syncthreads();
        if (s_abort) break;
        const int chunk = cc;
        cq++;
        next_phase(cc, cp);
        next_phase(c1, p1);
        next_phase(c2, p2);
        mc = mn;
        mn = mnn;
#pragma unroll
        for (int kt = 0; kt < KT; kt++)
#pragma unroll
            for (int nt = 0; nt < NT; nt++) bcur[kt][nt] = bnxt[kt][nt];
        if (MODE == 0 && cc != chunk) {
            // add the finished chunk's image to y (Dirichlet rows skipped) and
            // leave the image zero for the next chunk
            const int nb0 = a.ch_np[chunk], n = (a.ch_np[chunk + 1] - nb0) * NVL;
            for (int i = threadIdx.x; i < n; i += blockDim.x) {
                const int ln = i / NVL, rem = i - ln * NVL, comp = rem / KB, cs = rem - comp * KB;
                const int nd = a.ch_nodes[nb0 + ln];
                const long dof = 3L * (nd & 0x1FFFFFFF) + comp;
                if (!((nd >> (29 + comp)) & 1)) atomicAdd(&y[dof * KB + cs], yl[i]);
                yl[i] = 0.0;
            }
            __syncthreads();
        }
    }
    // on an abort, let this warp's copies in flight land before the CTA exits
    if (lane == 0 && pending) {
        for (int s = 0; s < ST; s++)
            if ((pending >> s) & 1u) mbar_wait(&bar[warp * ST + s], (parity >> s) & 1u, a.wait_cycles);
    }
}

// ----------------------------------------------------------------- block vector helpers
// dst[dof*kb + k] = src[k*n + dof] (k < ncase), 0 for padded cases
template <class TS, class TD>
__global__ void k_interleave(long n, int ncase, int kb, const TS* __restrict__ src, TD* __restrict__ dst) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n * kb; i += (long)gridDim.x * blockDim.x) {
        const long dof = i / kb;
        const int k = (int)(i - dof * kb);
        dst[i] = k < ncase ? (TD)src[(size_t)k * n + dof] : TD(0);
    }
}
template <class TS, class TD>
__global__ void k_deinterleave(long n, int ncase, int kb, const TS* __restrict__ src, TD* __restrict__ dst) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n * ncase; i += (long)gridDim.x * blockDim.x) {
        const int k = (int)(i / n);
        const long dof = i - (long)k * n;
        dst[i] = (TD)src[dof * kb + k];
    }
}
// Dirichlet rows of a block result: y = beta b + alpha u on fixed DOFs
template <class TU>
__global__ void k_blk_fix_rows(int nf, int kb, const int* __restrict__ fixed, const TU* __restrict__ u,
                               double* __restrict__ y, const double* __restrict__ b, double alpha, double beta) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nf * kb) return;
    const long o = (long)fixed[i / kb] * kb + (i % kb);
    y[o] = (b ? beta * b[o] : 0.0) + alpha * (double)u[o];
}
__global__ void k_blk_init(long n, double* __restrict__ y, const double* __restrict__ b) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        y[i] = b ? b[i] : 0.0;
}

// ----------------------------------------------------------------- host entry points
static size_t blk_smem(int npk, int kb, int nodes, int stages) {
    return 128 * ((kWarps * stages * 8 + 127) / 128) +
           sizeof(double) * ((size_t)kWarps * stages * npk + (size_t)nodes * 3 * kb);
}

int blk_width(int ncases) { return ncases <= 4 ? 4 : ncases <= 8 ? 8 : 16; }

template <int NEN, int KB, int MODE, class TU, int ST>
static int launch_blk_st(Ctx& c, const TU* u, double* y, double alpha, double* uku) {
    BlockState& B = c.blk;
    auto kern = k_blk_kmv<NEN, KB, MODE, TU, ST>;
    const size_t smem = blk_smem(c.npk, KB, B.max_nodes, ST);
    TCK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int occ = 0;
    TCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kWarps * 32, smem));
    int dev = 0, nsm = 148;
    TCK(cudaGetDevice(&dev));
    TCK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int per_sm = c.tune.blk_ctas > 0 ? std::min(std::max(1, occ), c.tune.blk_ctas) : std::max(1, occ);
    const int grid = std::max(1, std::min(B.nchunks, per_sm * nsm));
    BlkArgs a{B.nchunks, B.ch_ph.p, B.ph_sl.p, B.ch_np.p, B.ch_nodes.p, B.sl_elem.p, B.sl_gn.p, B.sl_lc.p,
              B.sl_mask.p, B.keb.p, B.kperm.p, B.Es.p, B.max_nodes, B.err.p, c.wait.copy_cycles, c.wait.hold};
    kern<<<grid, kWarps * 32, smem, c.s>>>(a, u, y, alpha, uku), note_launch();
    TCK(cudaGetLastError());
    return 0;
}

template <int NEN, int KB, int MODE, class TU>
static int launch_blk(Ctx& c, const TU* u, double* y, double alpha, double* uku) {
    const int st = c.p.blk_stages ? c.p.blk_stages : c.tune.blk_stages;
    if (st == 2) return launch_blk_st<NEN, KB, MODE, TU, 2>(c, u, y, alpha, uku);
    return launch_blk_st<NEN, KB, MODE, TU, 3>(c, u, y, alpha, uku);
}

template <int MODE, class TU>
static int dispatch_blk(Ctx& c, const TU* u, double* y, double alpha, double* uku) {
    const int kb = c.blk.kb;
    if (c.nen == 8) {
        if (kb == 4) return launch_blk<8, 4, MODE, TU>(c, u, y, alpha, uku);
        if (kb == 8) return launch_blk<8, 8, MODE, TU>(c, u, y, alpha, uku);
        return launch_blk<8, 16, MODE, TU>(c, u, y, alpha, uku);
    }
    if (kb == 4) return launch_blk<4, 4, MODE, TU>(c, u, y, alpha, uku);
    if (kb == 8) return launch_blk<4, 8, MODE, TU>(c, u, y, alpha, uku);
    return launch_blk<4, 16, MODE, TU>(c, u, y, alpha, uku);
}

// Build the chunk/phase schedule and the slot-ordered Ke copy (once per mesh).
int blk_setup(Ctx& c) {
    BlockState& B = c.blk;
    if (B.ready) return 0;
    B.kb = blk_width(c.ncases);
    const int node_cap = B.kb <= 8 ? 96 : 64;
    TRET(blk_build_schedule(c, node_cap));
    TRET(B.keb.alloc((size_t)c.ne * c.npk));
    TRET(B.Es.alloc(c.ne));
    B.es_gen = -1;
    std::vector<int> perm;
    blk_bank_perm(c.nde, perm);
    TRET(B.kperm.upload(perm, c.s));
    k_keb_gather<<<c.ne, 128, 0, c.s>>>(c.ne, c.npk, B.sl_elem.p, B.kperm.p, c.ke64.p, B.keb.p), note_launch();
    TCK(cudaGetLastError());
    TRET(B.err.alloc(1));
    TRET(B.err.zero(c.s));
    B.ready = true;
    return 0;
}

static int refresh_es(Ctx& c) {
    BlockState& B = c.blk;
    if (B.es_gen == c.moduli_gen) return 0;
    k_es_gather<<<(c.ne + 255) / 256, 256, 0, c.s>>>(c.ne, B.sl_elem.p, c.Ee64.p, B.Es.p), note_launch();
    TCK(cudaGetLastError());
    B.es_gen = c.moduli_gen;
    return 0;
}

// y = beta b + alpha K(E) u on block vectors (b may be null; fixed rows: identity)
template <class TU>
static int blk_apply_t(Ctx& c, const TU* u, double* y, const double* b, double alpha) {
    TRET(blk_setup(c));
    TRET(refresh_es(c));
    const long nv = (long)c.ndof * c.blk.kb;
    k_blk_init<<<grid_for(nv, 256), 256, 0, c.s>>>(nv, y, b), note_launch();
    cudaEvent_t e0;
    prof_begin(c, PS_KMV, &e0);
    TRET((dispatch_blk<0, TU>(c, u, y, alpha, nullptr)));
    prof_end(c, PS_KMV, e0);
    const int nf = (int)c.fixed_h.size();
    if (nf)
        k_blk_fix_rows<TU><<<(nf * c.blk.kb + 255) / 256, 256, 0, c.s>>>(nf, c.blk.kb, c.fixed.p, u, y, b, alpha,
                                                                       1.0), note_launch();
    TCK(cudaGetLastError());
    return 0;
}
int blk_apply(Ctx& c, const double* u, double* y, const double* b, double alpha) {
    return blk_apply_t<double>(c, u, y, b, alpha);
}
int blk_apply_f32in(Ctx& c, const float* u, double* y, const double* b, double alpha) {
    return blk_apply_t<float>(c, u, y, b, alpha);
}
// uku[e] = sum over cases of u_e' Ke u_e for a block displacement
int blk_uku(Ctx& c, const double* u, double* uku) {
    TRET(blk_setup(c));
    return dispatch_blk<1, double>(c, u, nullptr, 1.0, uku);
}
int blk_interleave(Ctx& c, const double* src, double* dst) {
    const long n = c.ndof;
    k_interleave<double, double><<<grid_for(n * c.blk.kb, 256), 256, 0, c.s>>>(n, c.ncases, c.blk.kb, src, dst),
        note_launch();
    TCK(cudaGetLastError());
    return 0;
}
int blk_deinterleave(Ctx& c, const double* src, double* dst) {
    const long n = c.ndof;
    k_deinterleave<double, double><<<grid_for(n * c.ncases, 256), 256, 0, c.s>>>(n, c.ncases, c.blk.kb, src, dst),
        note_launch();
    TCK(cudaGetLastError());
    return 0;
}
int blk_check_error(Ctx& c) {
    if (!c.blk.err.p) return 0;
    int h = 0;
    TCK(cudaMemcpyAsync(&h, c.blk.err.p, sizeof(int), cudaMemcpyDeviceToHost, c.s));
    TCK(cudaStreamSynchronize(c.s));
    if (h) {
        // reported once; the flag is cleared so the context stays usable
        TCK(cudaMemsetAsync(c.blk.err.p, 0, sizeof(int), c.s));
        TCK(cudaStreamSynchronize(c.s));
        set_error("block operator: a TMA copy did not complete in time");
        return TOPO_ERR_TIMEOUT;
    }
    return 0;
}

}  // namespace topo
