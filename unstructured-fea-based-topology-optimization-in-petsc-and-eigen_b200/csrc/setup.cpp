// setup.cpp -- host-side builders run once per mesh: validation, device
// layouts of the connectivity (AoSoA tiles of 32 elements), boundary masks,
// node graph, and the geometry-only part of the smoothed-aggregation AMG
// hierarchy (aggregates, tentative prolongators, symbolic Galerkin patterns).
// Only the numeric Galerkin products are recomputed per design iteration
// (on the device).
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <atomic>
#include <mutex>
#include <thread>

#include "ctx.h"

namespace topo {

// ----------------------------------------------------------------- errors
static thread_local std::string g_err;

void set_error(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
}
const char* last_error() { return g_err.c_str(); }

long& launch_counter() {
    static long n = 0;
    return n;
}

int cuda_fail(cudaError_t e, const char* file, int line) {
    set_error("CUDA error %s (%s) at %s:%d", cudaGetErrorName(e), cudaGetErrorString(e), file, line);
    return e == cudaErrorMemoryAllocation ? TOPO_ERR_OOM : TOPO_ERR_CUDA;
}

// ----------------------------------------------------------------- host threads
// body(t) for t in [0, nth) on nth threads; if a thread cannot be started,
// the started ones are joined before the error propagates (the callers'
// GUARD turns it into an error return).
template <class F>
static void run_threads(int nth, F&& body) {
    std::vector<std::thread> th;
    try {
        for (int t = 0; t < nth; t++) th.emplace_back(body, t);
    } catch (...) {
        for (auto& x : th) x.join();
        throw;
    }
    for (auto& x : th) x.join();
}

// ----------------------------------------------------------------- product plans
// Pairs of C = A B per C block for the device's output-stationary product.
// Each pair holds the A block's slot in its row with the B row's length, and
// the offset of the B block's first value in the slot-interleaved B array
// (bkc values per block), so the device reads both blocks without looking
// up A's column or B's row pointer.
// block_index: each pair's B entry is the B block's index (B stored block by
// block, padded, see k_spgemm_plan's BL); otherwise the offset of the block's
// first value in the slot-interleaved layout
int build_plan(const Pattern& A, const Pattern& B, const Pattern& C, int bkc, ProductPlan& out, cudaStream_t s,
               bool block_index) {
    const int n = A.nrows;
    std::vector<int> ptr((size_t)C.nnzb() + 1, 0);
    const int nth = std::max(1, std::min(16, (int)std::thread::hardware_concurrency()));
    auto for_rows = [&](auto&& fn) {
        run_threads(nth, [&](int t) {
            std::vector<int> slot(C.ncols, -1);
            for (int i = (int)((long)n * t / nth); i < (int)((long)n * (t + 1) / nth); i++) fn(i, slot);
        });
    };
    std::atomic<bool> bad(false);
    // pass 1: pairs per C block
    for_rows([&](int i, std::vector<int>& slot) {
        for (int q = C.rp[i]; q < C.rp[i + 1]; q++) slot[C.ci[q]] = q;
        const int na = A.rp[i + 1] - A.rp[i];
        if (na > 65535) bad = true;
        for (int a = 0; a < na; a++) {
            const int k = A.ci[A.rp[i] + a];
            const int nb = B.rp[k + 1] - B.rp[k];
            if (nb > 65535 || ((size_t)B.rp[k + 1] * bkc) >> 32) bad = true;
            for (int sb = 0; sb < nb; sb++) {
                const int q = slot[B.ci[B.rp[k] + sb]];
                if (q < 0) { bad = true; continue; }
                ptr[q + 1]++;
            }
        }
        for (int q = C.rp[i]; q < C.rp[i + 1]; q++) slot[C.ci[q]] = -1;
    });
    if (bad) { set_error("product plan: a row is too long or a pattern is inconsistent"); return TOPO_ERR_UNSUPPORTED; }
    for (size_t q = 0; q + 1 < ptr.size(); q++) ptr[q + 1] += ptr[q];
    std::vector<uint2> pr((size_t)ptr.back());
    std::vector<int> fill(ptr.begin(), ptr.end() - 1);
    // pass 2: the pairs, in (A slot, B slot) order within each C block
    for_rows([&](int i, std::vector<int>& slot) {
        for (int q = C.rp[i]; q < C.rp[i + 1]; q++) slot[C.ci[q]] = q;
        const int na = A.rp[i + 1] - A.rp[i];
        for (int a = 0; a < na; a++) {
            const int k = A.ci[A.rp[i] + a];
            const int nb = B.rp[k + 1] - B.rp[k];
            for (int sb = 0; sb < nb; sb++) {
                const int q = slot[B.ci[B.rp[k] + sb]];
                pr[fill[q]++] = make_uint2(((uint32_t)a << 16) | (uint32_t)nb,
                                           block_index ? (uint32_t)(B.rp[k] + sb)
                                                       : (uint32_t)((size_t)B.rp[k] * bkc + (size_t)sb));
            }
        }
        for (int q = C.rp[i]; q < C.rp[i + 1]; q++) slot[C.ci[q]] = -1;
    });
    out.avg_row = C.nrows ? (int)((C.nnzb() + C.nrows - 1) / C.nrows) : 1;
    out.avg_pairs = C.nnzb() ? (int)(pr.size() / (size_t)C.nnzb()) : 1;
    TRET(out.ptr.upload(ptr, s));
    TRET(out.pr.upload(pr, s));
    return 0;
}

// ----------------------------------------------------------------- patterns
// Rows [0, n) split over up to 16 host threads; fn(i, mark) with a per-thread
// scratch array of `width` ints set to -1.
template <class F>
static void for_rows_mt(int n, int width, F&& fn) {
    const int nth = std::max(1, std::min({16, (int)std::thread::hardware_concurrency(), n / 4096 + 1}));
    run_threads(nth, [&](int t) {
        std::vector<int> mark(width, -1);
        for (int i = (int)((long)n * t / nth); i < (int)((long)n * (t + 1) / nth); i++) fn(i, mark);
    });
}

// Pattern of A B, each row's columns sorted: a counting pass and a filling
// pass over the rows, both split over host threads (the rows are
// independent, so the result does not depend on the split).
Pattern sym_spgemm(const Pattern& A, const Pattern& B) {
    Pattern C;
    C.nrows = A.nrows;
    C.ncols = B.ncols;
    C.rp.assign(A.nrows + 1, 0);
    for_rows_mt(A.nrows, B.ncols, [&](int i, std::vector<int>& mark) {
        int cnt = 0;
        for (int p = A.rp[i]; p < A.rp[i + 1]; p++) {
            const int k = A.ci[p];
            for (int q = B.rp[k]; q < B.rp[k + 1]; q++)
                if (mark[B.ci[q]] != i) {
                    mark[B.ci[q]] = i;
                    cnt++;
                }
        }
        C.rp[i + 1] = cnt;
    });
    for (int i = 0; i < A.nrows; i++) C.rp[i + 1] += C.rp[i];
    C.ci.resize(C.rp[A.nrows]);
    for_rows_mt(A.nrows, B.ncols, [&](int i, std::vector<int>& mark) {
        int w = C.rp[i];
        for (int p = A.rp[i]; p < A.rp[i + 1]; p++) {
            const int k = A.ci[p];
            for (int q = B.rp[k]; q < B.rp[k + 1]; q++)
                if (mark[B.ci[q]] != i) {
                    mark[B.ci[q]] = i;
                    C.ci[w++] = B.ci[q];
                }
        }
        std::sort(C.ci.begin() + C.rp[i], C.ci.begin() + w);
    });
    return C;
}

Pattern sym_transpose(const Pattern& A, std::vector<int>& perm) {
    Pattern T;
    T.nrows = A.ncols;
    T.ncols = A.nrows;
    T.rp.assign(T.nrows + 1, 0);
    long nnz = A.nnzb();
    for (long q = 0; q < nnz; q++) T.rp[A.ci[q] + 1]++;
    for (int i = 0; i < T.nrows; i++) T.rp[i + 1] += T.rp[i];
    T.ci.resize(nnz);
    perm.resize(nnz);
    std::vector<int> pos(T.rp.begin(), T.rp.end() - 1);
    for (int i = 0; i < A.nrows; i++)
        for (int q = A.rp[i]; q < A.rp[i + 1]; q++) {
            int t = pos[A.ci[q]]++;
            T.ci[t] = i;
            perm[t] = q;
        }
    return T;
}

// Greedy aggregation of a node graph (rows sorted, self included):
// phase 1 roots an aggregate at every node whose non-excluded neighbourhood
// is still untouched and takes the whole neighbourhood; phase 2 attaches
// each leftover node to the phase-1 aggregate of its first aggregated
// neighbour; phase 3 turns what remains into singletons.  Excluded nodes
// (all DOFs Dirichlet) belong to no aggregate (-1 on output).
int aggregate_graph(int nn, const std::vector<int>& rp, const std::vector<int>& ci, const unsigned char* excl,
                    std::vector<int>& agg) {
    agg.assign(nn, -1);
    for (int i = 0; i < nn; i++)
        if (excl && excl[i]) agg[i] = -2;
    int na = 0;
    for (int i = 0; i < nn; i++) {
        if (agg[i] != -1) continue;
        bool ok = true;
        for (int p = rp[i]; p < rp[i + 1]; p++) {
            int j = ci[p];
            if (j != i && agg[j] >= 0) { ok = false; break; }
        }
        if (!ok) continue;
        for (int p = rp[i]; p < rp[i + 1]; p++) {
            int j = ci[p];
            if (agg[j] == -1) agg[j] = na;
        }
        agg[i] = na;
        na++;
    }
    std::vector<int> a1(agg);
    for (int i = 0; i < nn; i++) {
        if (a1[i] != -1) continue;
        for (int p = rp[i]; p < rp[i + 1]; p++) {
            int j = ci[p];
            if (a1[j] >= 0) { agg[i] = a1[j]; break; }
        }
    }
    for (int i = 0; i < nn; i++)
        if (agg[i] == -1) agg[i] = na++;
    for (int i = 0; i < nn; i++)
        if (agg[i] == -2) agg[i] = -1;
    return na;
}

// Node graph (each row: the nodes sharing an element with it, itself
// included, sorted) = block pattern of K.  Counting and filling passes over
// the rows split across host threads; an isolated node keeps its diagonal.
Pattern node_graph(int nn, int ne, int nen, const int32_t* element, const std::vector<int>& n2e_ptr,
                   const std::vector<int>& n2e) {
    (void)ne;
    Pattern G;
    G.nrows = G.ncols = nn;
    G.rp.assign(nn + 1, 0);
    for_rows_mt(nn, nn, [&](int i, std::vector<int>& mark) {
        int cnt = 0;
        for (int p = n2e_ptr[i]; p < n2e_ptr[i + 1]; p++) {
            const int e = n2e[p] / nen;
            for (int l = 0; l < nen; l++) {
                const int j = element[(long)e * nen + l];
                if (mark[j] != i) { mark[j] = i; cnt++; }
            }
        }
        G.rp[i + 1] = cnt ? cnt : 1;
    });
    for (int i = 0; i < nn; i++) G.rp[i + 1] += G.rp[i];
    G.ci.resize(G.rp[nn]);
    for_rows_mt(nn, nn, [&](int i, std::vector<int>& mark) {
        int w = G.rp[i];
        for (int p = n2e_ptr[i]; p < n2e_ptr[i + 1]; p++) {
            const int e = n2e[p] / nen;
            for (int l = 0; l < nen; l++) {
                const int j = element[(long)e * nen + l];
                if (mark[j] != i) { mark[j] = i; G.ci[w++] = j; }
            }
        }
        if (w == G.rp[i]) G.ci[w++] = i;
        std::sort(G.ci.begin() + G.rp[i], G.ci.begin() + w);
    });
    return G;
}

// For every element and pair of its local nodes (p, q): the slot of node q in
// node p's row of G (elements split across host threads).
std::vector<uint16_t> block_positions(int ne, int nen, const int32_t* element, const Pattern& G) {
    std::vector<uint16_t> bpos((size_t)ne * nen * nen);
    for_rows_mt(ne, 1, [&](int e, std::vector<int>&) {
        for (int p = 0; p < nen; p++) {
            const int np = element[(long)e * nen + p];
            const int* b = G.ci.data() + G.rp[np];
            const int len = G.rp[np + 1] - G.rp[np];
            for (int q = 0; q < nen; q++) {
                const int nq = element[(long)e * nen + q];
                bpos[((size_t)e * nen + p) * nen + q] = (uint16_t)(std::lower_bound(b, b + len, nq) - b);
            }
        }
    });
    return bpos;
}

// ----------------------------------------------------------------- mesh
int build_mesh(Ctx& c, const double* vertex, const int32_t* element, int n_fixed, const int32_t* fixed, int n_cases,
               const int32_t* case_ptr, const int32_t* load_dofs, const double* load_vals) {
    const int nen = c.nen, nn = c.nn, ne = c.ne;
    c.nde = 3 * nen;
    c.npk = c.nde * (c.nde + 1) / 2;
    c.nkf = nen * (nen + 1) / 2;
    c.ndof = 3 * nn;
    c.ntiles = (ne + 31) / 32;
    c.ncases = n_cases;
    for (long q = 0; q < 3L * nn; q++)
        if (!std::isfinite(vertex[q])) { set_error("vertex %ld is not finite", q / 3); return TOPO_ERR_MESH; }
    for (long q = 0; q < (long)ne * nen; q++)
        if (element[q] < 0 || element[q] >= nn) {
            set_error("element %ld references node %d outside [0,%d)", q / nen, element[q], nn);
            return TOPO_ERR_MESH;
        }
    for (int i = 0; i < n_fixed; i++)
        if (fixed[i] < 0 || fixed[i] >= c.ndof) { set_error("fixed DOF %d out of range", fixed[i]); return TOPO_ERR_MESH; }
    if (case_ptr[0] != 0) { set_error("case_ptr[0] must be 0"); return TOPO_ERR_ARG; }
    for (int k = 0; k < n_cases; k++) {
        if (case_ptr[k + 1] < case_ptr[k]) { set_error("case_ptr not monotone"); return TOPO_ERR_ARG; }
        for (int q = case_ptr[k]; q < case_ptr[k + 1]; q++) {
            if (load_dofs[q] < 0 || load_dofs[q] >= c.ndof) { set_error("load DOF %d out of range", load_dofs[q]); return TOPO_ERR_MESH; }
            if (!std::isfinite(load_vals[q])) { set_error("load value %d not finite", q); return TOPO_ERR_MESH; }
        }
    }
    c.vertex_h.assign(vertex, vertex + 3L * nn);
    c.elem_h.assign(element, element + (long)ne * nen);
    c.fixed_h.assign(fixed, fixed + n_fixed);
    c.dof_fixed_h.assign(c.ndof, 0);
    for (int i = 0; i < n_fixed; i++) c.dof_fixed_h[fixed[i]] = 1;

    cudaStream_t s = c.s;
    // AoSoA connectivity tiles + fixed masks
    std::vector<int> conn((size_t)c.ntiles * nen * 32, 0);
    std::vector<uint32_t> emask(ne, 0);
    for (int e = 0; e < ne; e++) {
        int t = e >> 5, lane = e & 31;
        uint32_t m = 0;
        for (int l = 0; l < nen; l++) {
            int nd = element[(long)e * nen + l];
            conn[((size_t)t * nen + l) * 32 + lane] = nd;
            for (int cc = 0; cc < 3; cc++)
                if (c.dof_fixed_h[3 * nd + cc]) m |= 1u << (cc * nen + l);
        }
        emask[e] = m;
    }
    TRET(c.conn.upload(conn, s));
    TRET(c.emask.upload(emask, s));
    TRET(c.elem.upload(c.elem_h, s));
    TRET(c.vertex.upload(c.vertex_h, s));
    TRET(c.dof_fixed.upload(c.dof_fixed_h, s));
    TRET(c.fixed.upload(c.fixed_h, s));

    // load vectors: VecSetValues(INSERT) then fixed DOFs zeroed (SolveFem.cpp:277-282,324-333)
    std::vector<double> F((size_t)n_cases * c.ndof, 0.0);
    for (int k = 0; k < n_cases; k++) {
        for (int q = case_ptr[k]; q < case_ptr[k + 1]; q++) F[(size_t)k * c.ndof + load_dofs[q]] = load_vals[q];
        for (int i = 0; i < n_fixed; i++) F[(size_t)k * c.ndof + fixed[i]] = 0.0;
    }
    TRET(c.F.upload(F, s));

    // node -> element incidence
    std::vector<int> n2e_ptr(nn + 1, 0), n2e((size_t)ne * nen);
    for (long q = 0; q < (long)ne * nen; q++) n2e_ptr[element[q] + 1]++;
    for (int i = 0; i < nn; i++) n2e_ptr[i + 1] += n2e_ptr[i];
    {
        std::vector<int> pos(n2e_ptr.begin(), n2e_ptr.end() - 1);
        for (long q = 0; q < (long)ne * nen; q++) n2e[pos[element[q]]++] = (int)q;
    }
    // node graph (self included, sorted) = block pattern of K
    Pattern G = node_graph(nn, ne, nen, element, n2e_ptr, n2e);
    c.maxdeg = G.max_row();
    if (c.maxdeg > 65535) { set_error("node degree too large"); return TOPO_ERR_MESH; }
    std::vector<uint16_t> bpos = block_positions(ne, nen, element, G);
    TRET(c.n2e_ptr.upload(n2e_ptr, s));
    TRET(c.n2e.upload(n2e, s));
    TRET(c.bpos.upload(bpos, s));

    c.hl.clear();
    c.hl.emplace_back();
    c.hl[0].bs = 3;
    c.hl[0].nnode = nn;
    c.hl[0].A = std::move(G);
    return 0;
}

// ----------------------------------------------------------------- AMG hierarchy (geometry only)
// Tentative prolongator: per aggregate, modified Gram-Schmidt on the rows of
// the near-null space (rigid-body modes about the aggregate centroid at
// level 0; the previous level's R factors above), Dirichlet rows dropped.
static void tentative(const Ctx& c, int lvl, const AmgHostLevel& L, const std::vector<double>& Bprev,
                      std::vector<double>& Pt, std::vector<double>& Bnext) {
    const int bs = L.bs, nnode = L.nnode, na = L.nagg;
    Pt.assign((size_t)nnode * bs * 6, 0.0);
    Bnext.assign((size_t)na * 6 * 6, 0.0);
    std::vector<int> cnt(na + 1, 0), mem;
    for (int i = 0; i < nnode; i++)
        if (L.agg[i] >= 0) cnt[L.agg[i] + 1]++;
    for (int a = 0; a < na; a++) cnt[a + 1] += cnt[a];
    mem.resize(cnt[na]);
    {
        std::vector<int> fill(cnt.begin(), cnt.end() - 1);
        for (int i = 0; i < nnode; i++)
            if (L.agg[i] >= 0) mem[fill[L.agg[i]]++] = i;
    }
    // aggregates are independent (disjoint rows of Pt, their own rows of
    // Bnext): split over host threads, which also overlaps the scattered
    // reads of member coordinates
    const int nth = std::max(1, std::min({16, (int)std::thread::hardware_concurrency(), na / 512 + 1}));
    auto work = [&](int a_begin, int a_end) {
    std::vector<double> Q;
    std::vector<long> rid;
    for (int a = a_begin; a < a_end; a++) {
        int m0 = cnt[a], m1 = cnt[a + 1];
        Q.clear();
        rid.clear();
        double cen[3] = {0, 0, 0};
        if (lvl == 0) {
            for (int t = m0; t < m1; t++)
                for (int q = 0; q < 3; q++) cen[q] += c.vertex_h[3 * (size_t)mem[t] + q];
            for (int q = 0; q < 3; q++) cen[q] /= (double)(m1 - m0);
        }
        for (int t = m0; t < m1; t++) {
            int i = mem[t];
            for (int q = 0; q < bs; q++) {
                long row = (long)bs * i + q;
                if (lvl == 0 && c.dof_fixed_h[row]) continue;
                rid.push_back((long)i * bs + q);
                if (lvl == 0) {
                    double x = c.vertex_h[3 * (size_t)i] - cen[0], y = c.vertex_h[3 * (size_t)i + 1] - cen[1],
                           z = c.vertex_h[3 * (size_t)i + 2] - cen[2];
                    const double rb[3][6] = {{1, 0, 0, -y, 0, z}, {0, 1, 0, x, -z, 0}, {0, 0, 1, 0, y, -x}};
                    for (int j = 0; j < 6; j++) Q.push_back(rb[q][j]);
                } else {
                    for (int j = 0; j < 6; j++) Q.push_back(Bprev[(size_t)row * 6 + j]);
                }
            }
        }
        int rows = (int)rid.size();
        double R[36] = {0};
        for (int j = 0; j < 6; j++) {
            double n0 = 0.0;
            for (int r = 0; r < rows; r++) n0 += Q[r * 6 + j] * Q[r * 6 + j];
            n0 = std::sqrt(n0);
            for (int i2 = 0; i2 < j; i2++) {
                double h = 0.0;
                for (int r = 0; r < rows; r++) h += Q[r * 6 + i2] * Q[r * 6 + j];
                R[i2 * 6 + j] = h;
                for (int r = 0; r < rows; r++) Q[r * 6 + j] -= h * Q[r * 6 + i2];
            }
            double nr = 0.0;
            for (int r = 0; r < rows; r++) nr += Q[r * 6 + j] * Q[r * 6 + j];
            nr = std::sqrt(nr);
            if (nr <= 1e-10 * n0 || nr == 0.0) {
                for (int r = 0; r < rows; r++) Q[r * 6 + j] = 0.0;
                R[j * 6 + j] = 0.0;
            } else {
                for (int r = 0; r < rows; r++) Q[r * 6 + j] /= nr;
                R[j * 6 + j] = nr;
            }
        }
        for (int r = 0; r < rows; r++)
            for (int j = 0; j < 6; j++) Pt[(size_t)rid[r] * 6 + j] = Q[r * 6 + j];
        for (int i2 = 0; i2 < 6; i2++)
            for (int j = 0; j < 6; j++) Bnext[((size_t)a * 6 + i2) * 6 + j] = R[i2 * 6 + j];
    }
    };
    run_threads(nth, [&](int t) { work((int)((long)na * t / nth), (int)((long)na * (t + 1) / nth)); });
}

int build_amg_host(Ctx& c) {
    const topo_params& p = c.p;
    std::vector<unsigned char> excl(c.nn, 0);
    for (int i = 0; i < c.nn; i++)
        excl[i] = c.dof_fixed_h[3 * i] && c.dof_fixed_h[3 * i + 1] && c.dof_fixed_h[3 * i + 2];
    std::vector<double> B, Bnext;
    int maxlev = std::min(std::max(p.amg_max_levels, 1), kMaxLevels);
    for (int lvl = 0;; lvl++) {
        AmgHostLevel& L = c.hl[lvl];
        long ndof = (long)L.nnode * L.bs;
        if (lvl + 1 >= maxlev || ndof <= p.amg_coarse_max) break;
        L.nagg = aggregate_graph(L.nnode, L.A.rp, L.A.ci, lvl == 0 ? excl.data() : nullptr, L.agg);
        if (L.nagg == 0 || L.nagg >= L.nnode) { L.agg.clear(); L.nagg = 0; break; }
        tentative(c, lvl, L, B, L.Pt, Bnext);
        Pattern Ptp;
        Ptp.nrows = L.nnode;
        Ptp.ncols = L.nagg;
        Ptp.rp.assign(L.nnode + 1, 0);
        for (int i = 0; i < L.nnode; i++) {
            Ptp.rp[i + 1] = Ptp.rp[i] + (L.agg[i] >= 0 ? 1 : 0);
            if (L.agg[i] >= 0) Ptp.ci.push_back(L.agg[i]);
        }
        L.P = p.amg_smooth_p ? sym_spgemm(L.A, Ptp) : Ptp;
        L.ptpos.assign(L.nnode, -1);
        for (int i = 0; i < L.nnode; i++) {
            if (L.agg[i] < 0) continue;
            const int* b = L.P.ci.data() + L.P.rp[i];
            int len = L.P.rp[i + 1] - L.P.rp[i];
            const int* f = std::lower_bound(b, b + len, L.agg[i]);
            L.ptpos[i] = (f != b + len && *f == L.agg[i]) ? (int)(f - b) : -1;
        }
        L.AP = sym_spgemm(L.A, L.P);
        L.R = sym_transpose(L.P, L.rperm);
        AmgHostLevel next;
        next.bs = 6;
        next.nnode = L.nagg;
        next.A = sym_spgemm(L.R, L.AP);
        B.swap(Bnext);
        c.hl.push_back(std::move(next));
    }
    c.nlev = (int)c.hl.size();
    // upload
    cudaStream_t s = c.s;
    for (int l = 0; l < c.nlev; l++) {
        AmgHostLevel& H = c.hl[l];
        AmgDevLevel& D = c.dl[l];
        D.bs = H.bs;
        D.nnode = H.nnode;
        D.ndof = H.nnode * H.bs;
        D.nagg = H.nagg;
        TRET(D.A.upload(H.A, s));
        std::vector<int> dp(H.nnode, -1);
        for (int i = 0; i < H.nnode; i++)
            for (int q = H.A.rp[i]; q < H.A.rp[i + 1]; q++)
                if (H.A.ci[q] == i) dp[i] = q - H.A.rp[i];
        for (int i = 0; i < H.nnode; i++)
            if (dp[i] < 0) { set_error("AMG level %d row %d has no diagonal block", l, i); return TOPO_ERR_MESH; }
        TRET(D.diagpos.upload(dp, s));
        if (l == 0) {
            // sliced ELLPACK: slice width = longest row of the 32-row slice,
            // padding blocks point at the row itself with zero values
            D.nslices = (H.nnode + 31) / 32;
            std::vector<int> sp(D.nslices + 1, 0), sci;
            for (int sl = 0; sl < D.nslices; sl++) {
                int w = 0;
                for (int r = 32 * sl; r < std::min(H.nnode, 32 * sl + 32); r++) w = std::max(w, H.A.rp[r + 1] - H.A.rp[r]);
                sp[sl + 1] = sp[sl] + 32 * w;
            }
            sci.assign(sp[D.nslices], 0);
            for (int sl = 0; sl < D.nslices; sl++) {
                int w = (sp[sl + 1] - sp[sl]) / 32;
                for (int ln = 0; ln < 32; ln++) {
                    int r = 32 * sl + ln;
                    for (int k = 0; k < w; k++) {
                        int col = r < H.nnode ? r : 0;
                        if (r < H.nnode && k < H.A.rp[r + 1] - H.A.rp[r]) col = H.A.ci[H.A.rp[r] + k];
                        sci[sp[sl] + 32 * k + ln] = col;
                    }
                }
            }
            D.sell_blocks = sp[D.nslices];
            TRET(D.sell_ptr.upload(sp, s));
            TRET(D.sell_ci.upload(sci, s));
        }
        if (l + 1 < c.nlev) {
            TRET(D.P.upload(H.P, s));
            {
                // greedy packing of consecutive P rows into warps of <= 32 rows and <= 32 blocks
                std::vector<int> wr(1, 0);
                bool ok = true;
                int rows = 0, blocks = 0;
                for (int i = 0; i < H.P.nrows && ok; i++) {
                    const int nb = H.P.rp[i + 1] - H.P.rp[i];
                    if (nb > 32) ok = false;
                    if (rows == 32 || blocks + nb > 32) {
                        wr.push_back(i);
                        rows = 0;
                        blocks = 0;
                    }
                    rows++;
                    blocks += nb;
                }
                wr.push_back(H.P.nrows);
                D.pnw = 0;
                if (ok && H.P.nrows > 0) {
                    TRET(D.pwrow.upload(wr, s));
                    D.pnw = (int)wr.size() - 1;
                }
            }
            TRET(D.AP.upload(H.AP, s));
            TRET(D.R.upload(H.R, s));
            TRET(D.ptpos.upload(H.ptpos, s));
            TRET(D.rperm.upload(H.rperm, s));
            Pattern Ptp;
            Ptp.nrows = H.nnode;
            Ptp.ncols = H.nagg;
            Ptp.rp.assign(H.nnode + 1, 0);
            std::vector<double> pv;
            std::vector<float> pv32;
            for (int i = 0; i < H.nnode; i++) {
                Ptp.rp[i + 1] = Ptp.rp[i];
                if (H.agg[i] < 0) continue;
                Ptp.rp[i + 1]++;
                Ptp.ci.push_back(H.agg[i]);
                for (int q = 0; q < H.bs * 6; q++) {
                    pv.push_back(H.Pt[(size_t)i * H.bs * 6 + q]);
                    pv32.push_back((float)H.Pt[(size_t)i * H.bs * 6 + q]);
                }
            }
            TRET(D.Ptp.upload(Ptp, s));
            TRET(D.Pt64c.upload(pv, s));
            TRET(D.Pt32c.upload(pv32, s));
            {
                // the same blocks padded to whole 16-byte vectors (the B operand of A Pt)
                const int bb = H.bs * 6, b64 = (bb + 1) / 2 * 2, b32 = (bb + 3) / 4 * 4;
                const size_t nbk = pv.size() / bb;
                std::vector<double> q64(nbk * b64, 0.0);
                std::vector<float> q32(nbk * b32, 0.0f);
                for (size_t g = 0; g < nbk; g++)
                    for (int e = 0; e < bb; e++) {
                        q64[g * b64 + e] = pv[g * bb + e];
                        q32[g * b32 + e] = pv32[g * bb + e];
                    }
                TRET(D.Pt64p.upload(q64, s));
                TRET(D.Pt32p.upload(q32, s));
            }
            // B blocks are bs x 6 in all three products (Pt, P, A P)
            TRET(build_plan(H.A, Ptp, H.P, H.bs * 6, D.plan_T, s, true));  // B: Pt block by block
            TRET(build_plan(H.A, H.P, H.AP, H.bs * 6, D.plan_AP, s, true));     // B: P block by block
            TRET(build_plan(H.R, H.AP, c.hl[l + 1].A, H.bs * 6, D.plan_RAP, s, true));  // B: A P block by block
        }
    }
    return 0;
}

}  // namespace topo
