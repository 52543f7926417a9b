// ctx.h -- internal state of one topology-optimisation job and the internal
// (C++) interface between the host-side builders and the device stages.
#pragma once
#include <cuda_runtime.h>

#include <array>
#include <cstdint>
#include <string>
#include <vector>

#include "common.cuh"

namespace topo {

constexpr int kMaxLevels = 8;
constexpr int kMaxM = 4;        // constraints supported by the device MMA
constexpr int kMaxCases = 16;   // load cases of the block solver

// Block-sparse pattern (host).  Values of the device copies are stored
// "slot-interleaved": entry e (0..BB-1) of the block in slot s of row i sits
// at val[rp[i]*BB + e*nb_i + s] with nb_i = rp[i+1]-rp[i], so a warp whose
// lanes walk the slots of one row reads each entry coalesced.
struct Pattern {
    int nrows = 0, ncols = 0;
    std::vector<int> rp, ci;
    long nnzb() const { return rp.empty() ? 0 : rp.back(); }
    int max_row() const {
        int m = 0;
        for (int i = 0; i < nrows; i++) m = std::max(m, rp[i + 1] - rp[i]);
        return m;
    }
};

struct DevPattern {
    int nrows = 0, ncols = 0, maxrow = 0;
    long nnzb = 0;
    DBuf<int> rp, ci;
    int upload(const Pattern& p, cudaStream_t s) {
        nrows = p.nrows; ncols = p.ncols; nnzb = p.nnzb(); maxrow = p.max_row();
        TRET(rp.upload(p.rp, s));
        TRET(ci.upload(p.ci, s));
        return 0;
    }
};

// Host-built, geometry-only hierarchy (aggregates, tentative prolongators,
// patterns of every Galerkin product).  Built once per mesh.
struct AmgHostLevel {
    int bs = 3;                 // DOFs per node at this level (3, then 6)
    int nnode = 0;
    Pattern A;                  // bs x bs blocks (level 0: mesh node graph)
    std::vector<int> agg;       // node -> aggregate, -1 none (excluded)
    int nagg = 0;
    std::vector<double> Pt;     // nnode x bs x 6 tentative prolongator blocks
    Pattern P;                  // pattern of A * Pt (= pattern of smoothed P)
    std::vector<int> ptpos;     // slot of agg(i) in P row i, -1 none
    Pattern AP;                 // pattern of A * P
    Pattern R;                  // P^T
    std::vector<int> rperm;     // R block -> P block index
};

// Output-stationary plan of a fixed-pattern block product C = A B: for every
// block of C (CSR order) the (A block, B block) pairs that contribute, each
// as {slot in A's row << 16 | length of B's row, B block}, the B block given
// as the offset of its first value (B slot-interleaved) or as its index (B
// stored block by block, padded).  Built on the host once per mesh.
struct ProductPlan {
    DBuf<int> ptr;              // nnzb(C) + 1
    DBuf<uint2> pr;             // pairs: {A slot << 16 | B row length, B block (offset or index)}
    int avg_row = 0;            // mean blocks per C row (picks lanes per row)
    int avg_pairs = 0;          // mean pairs per C block (picks lanes per block)
};
int build_plan(const Pattern& A, const Pattern& B, const Pattern& C, int bkc, ProductPlan& out, cudaStream_t s,
               bool block_index);

struct AmgDevLevel {
    int bs = 3, nnode = 0, ndof = 0, nagg = 0;
    DevPattern A, P, AP, R;
    DBuf<int> diagpos;          // slot of the diagonal block in each A row
    DBuf<int> ptpos, rperm;
    // level 0 only: sliced-ELLPACK (32-row slices) copy of A for the smoother;
    // block k of row 32s+l is entry sell_ptr[s] + 32k + l
    int nslices = 0;
    long sell_blocks = 0;
    DBuf<int> sell_ptr, sell_ci;
    ProductPlan plan_T, plan_AP, plan_RAP;  // A Pt, A P, R (A P)
    // prolongation with one block per lane: warp w owns the P rows
    // [pwrow[w], pwrow[w+1]) (at most 32 rows and 32 blocks); pnw = 0 when a
    // P row has more than 32 blocks
    DBuf<int> pwrow;
    int pnw = 0;
    DevPattern Ptp;             // tentative prolongator: one block per aggregated node
    DBuf<double> Pt64c;         // its bs x 6 blocks (compact, FP64)
    DBuf<float> Pt32c;          // (FP32 copy for the mixed form)
    DBuf<double> Pt64p;         // the same blocks padded to 16-byte vectors (B operand of A Pt)
    DBuf<float> Pt32p;
};

// numeric values of the hierarchy in precision T
template <class T>
struct AmgVals {
    DBuf<T> A[kMaxLevels], P[kMaxLevels], T_[kMaxLevels], R[kMaxLevels];
    DBuf<T> AP[kMaxLevels];     // A P block by block, padded (the B operand of R (A P))
    DBuf<T> dinv[kMaxLevels];
    DBuf<T> x[kMaxLevels], b[kMaxLevels], r[kMaxLevels], d[kMaxLevels], d2[kMaxLevels], t[kMaxLevels];
    DBuf<T> pv[kMaxLevels], pw[kMaxLevels];   // power-iteration vectors (warm start)
    DBuf<T> A0s;                // level-0 operator in the sliced-ELLPACK layout
    DBuf<T> Pk[kMaxLevels];     // P in the packed block-major layout (pk_off)
    DBuf<T> Pb[kMaxLevels];     // P block by block, each block padded to 16 bytes (the B operand of A P)
    DBuf<T> kst;                // node-row copy of the element matrices (k_ke_node_rows), built once
    bool allocated = false;
};

// mixed form, level 0 in FP16 on the diagonally scaled operator (amg.cu)
struct Half0 {
    DBuf<uint16_t> S;           // D^-1/2 A D^-1/2 as FP16, sliced-ELLPACK layout
    DBuf<float> s, sinv;        // D^1/2, D^-1/2 per DOF
    bool valid = false;         // built for the current design iteration
};

// CUDA graphs of the Arnoldi steps of one FGMRES form: step j (V-cycle,
// operator, Gram-Schmidt, Givens, residual read-back) is captured once and
// replayed in every later solve with the same buffers.  `sig` identifies the
// buffers and options the graphs were captured with; any change drops them.
struct StepGraphs {
    std::vector<cudaGraphExec_t> exec;
    std::vector<long> launches;      // kernels per replay (for the launch counter)
    uint64_t sig = 0;
    uint64_t seen = 0;               // signature of the previous solve (capture from the second on)
    cudaStream_t cap = nullptr;      // private capture stream (the context's may be the legacy one)
    bool disabled = false;           // capture failed once: direct launches from then on
    void drop() {
        for (auto e : exec)
            if (e) cudaGraphExecDestroy(e);
        exec.clear();
        launches.clear();
    }
    ~StepGraphs() {
        drop();
        if (cap) cudaStreamDestroy(cap);
    }
};
int step_graph_run(struct Ctx& c, StepGraphs& G, int j, bool capture_ok, int (*body)(struct Ctx&, void*), void* arg);
uint64_t sig_mix(uint64_t h, uint64_t v);

// block (KB right-hand sides) work vectors of the V-cycle
template <class T>
struct AmgBlkVecs {
    DBuf<T> x[kMaxLevels], b[kMaxLevels], r[kMaxLevels], d[kMaxLevels], d2[kMaxLevels], t[kMaxLevels];
    int kb = 0, nlev = 0;
};

// k-load block operator and solver state (block.cu, block_solve.cu)
struct BlockState {
    bool ready = false;
    int kb = 0;                 // case width of block vectors (4, 8 or 16)
    int nchunks = 0, nphases = 0, max_nodes = 0, max_phases = 0, node_cap = 0;
    DBuf<int> ch_ph, ph_sl, ch_np, ch_nodes;  // chunk -> phases, phase -> slots, chunk -> nodes
    DBuf<int> sl_elem, sl_gn;   // slot -> element, slot -> global nodes
    DBuf<uint16_t> sl_lc;       // slot -> chunk-local nodes
    DBuf<uint32_t> sl_mask;     // slot -> fixed local DOFs
    DBuf<double> keb;           // slot -> packed Ke (E = 1), entry k at kperm[k] (bank layout)
    DBuf<int> kperm;
    DBuf<double> Es;            // slot -> SIMP modulus of the current design
    int es_gen = -1;            // moduli generation Es was gathered from
    DBuf<int> err;              // set when a bounded wait expired
    // block FGMRES
    DBuf<double> F, U;          // loads and solutions, [dof][KB]
    DBuf<double> V, w, Z64;     // basis (m+1 block vectors), work, FP64 directions
    DBuf<float> Z32;            // FP32 directions (mixed form)
    DBuf<double> st;            // per-case Arnoldi states + scratch
    DBuf<int> ik;               // per-case active flags and column counts
    PinnedScalars hs;           // host mirror of the per-iteration outputs
    bool u_valid = false;       // U holds this run's previous block solution
    bool u_fresh = false;       // U belongs to the last displacement solve
    AmgBlkVecs<float> bv32;     // V-cycle work vectors, [dof][KB] per level
    AmgBlkVecs<double> bv64;
    StepGraphs graphs;          // captured Arnoldi steps of the block FGMRES
};

struct Ctx {
    topo_params p{};
    cudaStream_t s = nullptr;
    bool own_stream = false;

    // ---- mesh
    int nen = 8, nn = 0, ne = 0, ntiles = 0, ndof = 0, nde = 24, npk = 300, nkf = 36;
    int ncases = 1;
    std::vector<double> vertex_h;
    std::vector<int> elem_h, fixed_h;
    std::vector<unsigned char> dof_fixed_h;
    DBuf<int> conn;             // AoSoA [tile][nen][32]
    DBuf<int> elem;             // [ne][nen]
    DBuf<double> vertex;        // [nn][3]
    DBuf<uint32_t> emask;       // fixed local DOFs per element (bit c*nen+l)
    DBuf<unsigned char> dof_fixed;
    DBuf<int> fixed;
    DBuf<double> ke64;          // AoSoA [tile][npk][32], E = 1
    DBuf<float> ke32;
    DBuf<double> vol;
    double TV = 0.0;
    DBuf<double> F;             // [ncases][ndof]
    DBuf<int> n2e_ptr, n2e;     // node -> element*nen + local
    DBuf<double> det_scr;       // deterministic form: per-element operator contributions [tile][nde][32]
    DBuf<uint16_t> bpos;        // [ne][nen][nen] slot of node q in node p's row
    int maxdeg = 0;

    // ---- filter
    DBuf<double> kf;            // AoSoA [tile][nkf][32]
    DBuf<double> tf;            // AoSoA [tile][nen][32]
    DBuf<double> fdiag_inv, RX, TX, fr, fz, fp, fw;

    // ---- AMG
    std::vector<AmgHostLevel> hl;
    AmgDevLevel dl[kMaxLevels];
    int nlev = 0;
    DBuf<double> cinv;          // coarsest inverse (FP64, ncoarse^2)
    DBuf<double> cA;            // coarsest dense matrix scratch
    AmgVals<double> v64;
    AmgVals<float> v32;
    Half0 h0;
    DBuf<double> rho;           // [kMaxLevels] spectral estimates of D^-1 A
    bool amg_ready = false;

    // ---- displacement solve
    DBuf<double> Ee64;          // SIMP moduli of the current xphys
    int moduli_gen = 0;         // bumped whenever Ee64/Ee32 are recomputed
    DBuf<float> Ee32;
    DBuf<double> U;             // [ncases][ndof]
    DBuf<double> uku;           // per-element u'Ke u summed over cases
    DBuf<double> V;             // Krylov basis (restart+1) x ndof
    DBuf<double> Z64;           // preconditioned directions (FP64 form)
    DBuf<float> Z32;            // (mixed form)
    DBuf<double> w, wtmp;       // wtmp: device Arnoldi state + per-iteration outputs
    std::vector<cudaEvent_t> gm_ev;  // one per Arnoldi step (pipelined residual checks)
    StepGraphs graphs;          // captured Arnoldi steps of the single-load FGMRES
    DBuf<double> red;           // reduction partials
    DBuf<unsigned> red_count;   // blocks done of the last-block reduction in flight (0 between launches)
    DBuf<double> dsc;           // device scalars
    DBuf<int> di;               // device integers (DiSlot)
    PinnedScalars hsc;          // pinned host mirror for readbacks

    // ---- MMA (MMA.cpp state; the outer iteration k lives in di[DI_MMA_K])
    // bounds of the device-side waits (grid barrier spins, bulk-copy wait
    // cycles) and the test form that makes them run out (topo_test_wait_limits)
    struct WaitLimits {
        unsigned barrier_spins = 1u << 24;
        unsigned long long copy_cycles = 2000000000ull;  // about a second at 2 GHz
        int hold = 0;
    } wait;
    double asyminit = 0.5, asymdec = 0.7, asyminc = 1.2;
    int constraint_mod = 0, robust_type = 0;
    std::vector<double> a, c, d;
    DBuf<double> L, Uas, alpha, beta, p0, q0, pij, qij, xo1, xo2;
    DBuf<double> mma_scal;      // lam, mu, y, z, b ... device side
    DBuf<unsigned> bar;         // grid barrier words
    DBuf<int> bar_err;

    // ---- driver design vectors (OptPara)
    DBuf<double> X, Xold, XF, XP, dfdx, dgdx, xmin, xmax;
    int itr = 0;
    double ch = 1.0, beta_proj = 1.0, beta_tmp = 1.0;
    bool opt_ready = false;
    bool u_valid = false;       // U holds a solution of this optimisation run

    BlockState blk;

    // Device-driven design iteration (stepgraph.cu): the main.cpp loop body
    // captured as CUDA graphs, with the FGMRES and filter-CG loops run as
    // conditional graph nodes whose conditions are set on the device.
    struct StepGraph {
        bool dd = false;                 // capturing: stages take their device-driven form
        cudaStream_t cap = nullptr;      // top-level capture stream
        cudaStream_t body[4] = {};       // capture streams of nested conditional bodies
        int depth = 0;
        int coop_blocks = 0;             // capturing: cap on the dual solve's grid (0: one block per SM)
        // three graphs: [0] solve, sensitivities, filtered sensitivities, move
        // limits; [1] the MMA update (its cooperative dual solve) and the design
        // change; [2] filter, projection, results.  The part-1 graphs of all
        // contexts of a process run one after another on each device (the
        // dual solve's grid barrier wants its blocks resident together).
        cudaGraphExec_t exec[3] = {nullptr, nullptr, nullptr};
        long launches[3] = {0, 0, 0};    // kernels per replay (for the launch counter)
        cudaEvent_t p0_done = nullptr;   // recorded after part 0
        int stage = 0;                   // topo_opt_step_async: 0 idle, 1 part 0 in flight,
                                         // 2 parts 1-2 in flight, 3 a direct step finished
        int direct_rc = 0;               // its status
        uint64_t sig = 0;                // options and buffers the graphs were captured with
        uint64_t gen = 0;                // capture number (process-wide; batch graphs follow it)
        bool disabled = false;           // capture failed: direct launches from then on
        bool state_dirty = true;         // host itr/beta changed since the device copies
        DBuf<double> out;                // collected per-step results (read once per step)
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        void drop() {
            for (auto& e : exec) {
                if (e) cudaGraphExecDestroy(e);
                e = nullptr;
            }
        }
        ~StepGraph() {
            drop();
            if (cap) cudaStreamDestroy(cap);
            for (auto b : body)
                if (b) cudaStreamDestroy(b);
            for (auto e : {e0, e1, p0_done})
                if (e) cudaEventDestroy(e);
        }
    } sg;

    // launch shapes (autotuned at the first solve, see autotune.cu)
    struct Tune {
        int kmv_block = 128;        // k_kmv threads per block
        int sell_block = 256;       // level-0 sliced-ELLPACK kernels
        int sell_variant = 0;       // their row-product shape (k_sell_spmv's V)
        int red_blocks = 1184;      // grid of the vector reductions / Gram-Schmidt sweeps
        int blk_ctas = 0;           // block operator CTAs per SM (0: occupancy limit)
        int blk_stages = 3;         // block operator Ke copies in flight per warp (2 or 3)
        int blk_sell_u = 1;         // block level-0 sweep: slots per load group (1 or 3)
        int bsr_g[kMaxLevels] = {}; // lanes per block row of the level-l (>= 1) smoother/residual (0: by row length)
        bool single_done = false, block_done = false;
    } tune;

    topo_solve_info info{};
    bool vc_pdl = false;            // V-cycle kernels launched with programmatic dependent launch
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};

    // per-kernel CUDA-event timing of the hot kernels (off unless enabled)
    struct Prof {
        bool on = false;
        std::vector<cudaEvent_t> pool;                 // free events
        std::vector<std::pair<cudaEvent_t, cudaEvent_t>> rec[12];
    } prof;
};

// launch shapes are timed on the context's data unless the run must be
// bitwise reproducible (a shape can change the order of a sum)
inline bool tuning_on(const Ctx& c) { return c.p.autotune && !c.p.deterministic; }
// several load cases share the block operator and block V-cycle, unless the
// run must be bitwise reproducible (the block operator adds chunk images
// with atomics): then they are solved one by one
inline bool block_cases(const Ctx& c) { return c.ncases > 1 && c.p.fem_block && !c.p.deterministic; }

// profiler slots
enum ProfSlot {
    PS_KMV = 0, PS_CHEB0 = 1, PS_RES0 = 2, PS_FILTER = 3,
    PS_SETUP_ASM = 4,     // level-0 assembly + sliced-ELLPACK copy + diagonals
    PS_SETUP_RHO = 5,     // power iterations
    PS_SETUP_GAL = 6,     // smoothing of P + Galerkin products + transposes
    PS_SETUP_COARSE = 7,  // coarsest dense inverse
    PS_VCYCLE = 8,        // whole preconditioner application
    PS_VC_COARSE = 9,     // V-cycle below level 0 (from the level-0 restriction to the prolongation)
    PS_ORTH = 10,         // Gram-Schmidt sweeps of one Arnoldi step
    PS_SOLVE = 11,        // whole displacement solve (setup excluded)
    PS_COUNT = 12
};
cudaEvent_t prof_event(Ctx& c);
inline void prof_begin(Ctx& c, int slot, cudaEvent_t* e0) {
    *e0 = nullptr;
    if (c.prof.on) { *e0 = prof_event(c); cudaEventRecord(*e0, c.s); }
    (void)slot;
}
inline void prof_end(Ctx& c, int slot, cudaEvent_t e0) {
    if (!c.prof.on || !e0) return;
    cudaEvent_t e1 = prof_event(c);
    cudaEventRecord(e1, c.s);
    c.prof.rec[slot].push_back({e0, e1});
}

// ---- host builders (setup.cpp)
int build_mesh(Ctx& c, const double* vertex, const int32_t* element, int n_fixed, const int32_t* fixed,
               int n_cases, const int32_t* case_ptr, const int32_t* load_dofs, const double* load_vals);
int build_amg_host(Ctx& c);
int aggregate_graph(int nn, const std::vector<int>& rp, const std::vector<int>& ci,
                    const unsigned char* excl, std::vector<int>& agg);
Pattern sym_spgemm(const Pattern& A, const Pattern& B);
Pattern sym_transpose(const Pattern& A, std::vector<int>& perm);

// ---- device stages
int elem_setup(Ctx& c);                                            // kernels_elem.cu
int kmatvec(Ctx& c, const double* Ee, const double* u, double* y, int ncase = 1);
int kmatvec_f32in(Ctx& c, const double* Ee, const float* u, double* y);
int compute_moduli(Ctx& c, const double* xphys);
int fem_sensitivities(Ctx& c, const double* xphys, double* dfdx, double* dgdx);  // fx,gx -> dsc[0],[1]
int filter_tf(Ctx& c, const double* x, double* tx);
int filter_kf(Ctx& c, const double* r, double* y);
int filter_tfxT(Ctx& c, const double* rx, double* xf, bool clamp, double xmin);
int von_mises(Ctx& c, const double* xphys, double* vms);

int blk_width(int ncases);                                         // block.cu
int blk_bank_perm(int nd, std::vector<int>& perm);  // 1: conflict-free layout found, 0: identity
int blk_setup(Ctx& c);
int blk_apply(Ctx& c, const double* u, double* y, const double* b, double alpha);
int blk_apply_f32in(Ctx& c, const float* u, double* y, const double* b, double alpha);
int blk_uku(Ctx& c, const double* u, double* uku);
int blk_interleave(Ctx& c, const double* src, double* dst);
int blk_deinterleave(Ctx& c, const double* src, double* dst);
int blk_check_error(Ctx& c);

int amg_alloc(Ctx& c);                                             // amg.cu
int amg_numeric(Ctx& c);
int amg_level0_apply(Ctx& c, const void* x, void* y);
int amg_tune_levels(Ctx& c);  // lanes per block row of the levels >= 1, timed on the current hierarchy
int amg_reset_warm_start(Ctx& c);
int amg_level_copy(Ctx& c, int l, int which, std::vector<double>& vals_out, std::vector<int>& rp, std::vector<int>& ci,
                   int& nrows, int& ncols, int& br, int& bc);
int amg_vcycle64(Ctx& c, const double* b, double* x);
int amg_vcycle32(Ctx& c, const double* b64, float* x);

int autotune_single(Ctx& c);                                       // autotune.cu
int autotune_block(Ctx& c);
int fem_solve(Ctx& c, const double* xphys, double* u);             // solver.cu
int fem_solve_block(Ctx& c, const double* xphys, double* u);       // block_solve.cu
int filter_cg(Ctx& c, const double* b, double* x, int* its, int slot = 0);
int dev_dot(Ctx& c, const double* a, const double* b, long n, double* out_dev);
int finalize_sum(Ctx& c, const double* partials, int nparts, int nv, double* out_dev);

// conditional graph nodes (stepgraph.cu): the body is captured on a private
// stream (c.s is switched to it) until cond_end
int cond_begin(Ctx& c, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type);
int cond_end(Ctx& c);
int cond_handle(Ctx& c, cudaGraphConditionalHandle* h);  // handle on the graph being captured on c.s
// the device-driven step (stepgraph.cu): prepare (capture when needed) and
// say whether this step can be replayed; launch part p (0..2) on c.s; wait
// for the step and read its results
int opt_step_graph_prepare(Ctx& c, bool* ok);
int opt_step_graph_part(Ctx& c, int part);
int opt_step_graph_finish(Ctx& c);
int opt_step_graph_batch(Ctx* const* cs, int n, bool* launched);
void step_batch_forget(const Ctx* c);

int mma_alloc(Ctx& c);                                             // mma.cu
int mma_movelimit(Ctx& c, double Xmin, double Xmax, double movlim, const double* x, double* xmin, double* xmax);
int mma_update(Ctx& c, double* x, const double* dfdx, const double* gx_dev, const double* dgdx,
               const double* xmin, const double* xmax);
int mma_design_change(Ctx& c, const double* x, double* xold, double* ch_dev);
int mma_kkt(Ctx& c, const double* x, const double* dfdx, const double* gx_dev, const double* dgdx,
            const double* xmin, const double* xmax, double* n2, double* ninf);

// device scalar slots in Ctx::dsc
enum DscSlot {
    DS_FX = 0, DS_GX = 1,          // .. DS_GX + kMaxM - 1
    DS_CH = 8, DS_TMP = 9,
    DS_CG = 16,                    // CG scratch (16..31)
    DS_GM = 32,                    // FGMRES column (32..170)
    DS_KKT = 176,
    DS_TTOL = 180,                 // device-driven step: FGMRES stopping threshold
    DS_CGTOL = 181,                //   filter CG stopping threshold
    DS_RELRES = 182,               //   true relative residual of the last solve
    DS_BETA = 183, DS_BETA_TMP = 184,  // Heaviside beta state (PDEFilter.cpp:260-268)
    DS_COUNT = 200
};

// MMA scalars in Ctx::mma_scal: lam[4] mu[4] y[4] z b[4] its err
constexpr int kMmaSlots = 32;
enum { MS_LAM = 0, MS_MU = 4, MS_Y = 8, MS_Z = 12, MS_B = 13, MS_ITS = 17, MS_ERR = 18 };

// device integer slots in Ctx::di (the device-driven step's loop state, and
// the counters that live on the device in every form)
enum DiSlot {
    DI_ITS = 0, DI_KDONE = 1, DI_CONV = 2, DI_STOP = 3, DI_JMAX = 4,  // FGMRES
    DI_NAN = 5,                    // a solve met a non-finite residual
    DI_STATUS = 6,                 // FGMRES: 0 converged, 1 iteration cap
    DI_CG_ITS = 8,                 // filter CG iterations of solves 0..3
    DI_CG_STATUS = 12,             // filter CG status of solves 0..3
    DI_ITR = 16,                   // design iteration counter (main.cpp:72)
    DI_MMA_K = 17,                 // MMA outer iteration k (MMA.cpp:508)
    DI_CG_CUR = 18,                // iterations of the running filter CG
    DI_COUNT = 32
};

}  // namespace topo
