// stepgraph.cu -- the design iteration (main.cpp:72-112) replayed from CUDA graphs.
//
// A direct step (abi.cu opt_step) is driven by the host: it launches every
// kernel, reads the FGMRES residual after each Arnoldi step, reads the filter
// CG residual after each CG step and waits for the MMA dual solve.  Here the
// step is captured once into graphs in which those loops are conditional
// nodes (CUDA 12.4+): a WHILE node per solve, an IF node per Arnoldi step of
// an FGMRES cycle, and single-thread kernels that take the host's decisions
// on the device and set the nodes' conditions (cudaGraphSetConditional).
// Every loop is bounded by its solver's iteration cap.  A replayed step is
// three graph launches and one wait for its results; the same kernels run in
// the same order as in a direct step, so the results agree with a direct
// step to rounding.
//
// Several contexts (independent design instances) are advanced together by
// topo_opt_step_batch (abi.cu): the iterations of all replayable instances
// are one graph launch (opt_step_graph_batch below), each instance a branch
// of that graph; topo_opt_step_async and topo_opt_step_query let one host
// thread keep many instances going without waiting on any.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include "ctx.h"

namespace topo {

int fem_obj_sens_dev(Ctx& c, const double* xphys, double* dfdx, double* dgdx);
int filter_sens(Ctx& c, double* df, double* dg, int m);
int filter_apply(Ctx& c, const double* x, double* xf, double Xmin);
int heaviside(Ctx& c, const double* xf, double* xp, double x0, double beta0, double betamax, int itr, double Xmin,
              int proj);
int projected_sens(Ctx& c, const double* xf, double* df, double* dg, int m, double x0);
uint64_t sig_mix(uint64_t h, uint64_t v);
const char* last_error();

// ----------------------------------------------------------------- conditional nodes under stream capture
static int capture_graph_of(cudaStream_t s, cudaGraph_t* g, const cudaGraphNode_t** deps, size_t* nd) {
    cudaStreamCaptureStatus st;
    TCK(cudaStreamGetCaptureInfo(s, &st, nullptr, g, deps, nd));
    if (st != cudaStreamCaptureStatusActive) {
        set_error("internal: conditional node outside a stream capture");
        return TOPO_ERR_CUDA;
    }
    return 0;
}

int cond_handle(Ctx& c, cudaGraphConditionalHandle* h) {
    cudaGraph_t g;
    const cudaGraphNode_t* deps;
    size_t nd;
    TRET(capture_graph_of(c.s, &g, &deps, &nd));
    TCK(cudaGraphConditionalHandleCreate(h, g, 0, cudaGraphCondAssignDefault));
    return 0;
}

// Adds a conditional node after the work captured so far on c.s, and starts
// capturing its body on the private stream of the next nesting level (c.s
// names that stream until cond_end).
int cond_begin(Ctx& c, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type) {
    if (c.sg.depth >= 4) {
        set_error("internal: conditional nodes nested too deeply");
        return TOPO_ERR_CUDA;
    }
    cudaGraph_t g;
    const cudaGraphNode_t* deps;
    size_t nd;
    TRET(capture_graph_of(c.s, &g, &deps, &nd));
    cudaGraphNodeParams np = {cudaGraphNodeTypeConditional};
    np.conditional.handle = h;
    np.conditional.type = type;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    TCK(cudaGraphAddNode(&node, g, deps, nd, &np));
    TCK(cudaStreamUpdateCaptureDependencies(c.s, &node, 1, cudaStreamSetCaptureDependencies));
    cudaStream_t bs = c.sg.body[c.sg.depth];
    TCK(cudaStreamBeginCaptureToGraph(bs, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal));
    c.sg.depth++;
    c.s = bs;
    return 0;
}

int cond_end(Ctx& c) {
    if (c.sg.depth < 1) {
        set_error("internal: cond_end without cond_begin");
        return TOPO_ERR_CUDA;
    }
    cudaGraph_t g = nullptr;
    TCK(cudaStreamEndCapture(c.s, &g));
    c.sg.depth--;
    c.s = c.sg.depth ? c.sg.body[c.sg.depth - 1] : c.sg.cap;
    return 0;
}

// ----------------------------------------------------------------- step kernels
__global__ void k_itr_next(int* __restrict__ di) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        di[DI_ITR] += 1;
        di[DI_NAN] = 0;
    }
}

// The step's results in one place (read with one copy per step):
// [0] fx  [1..4] gx  [5] ch  [6] true relres  [7] beta  [8] beta_tmp
// [9] MMA inner iterations  [10] barrier timeout flag  [11] FGMRES its
// [12] FGMRES status  [13] NaN flag  [14..17] CG its  [18..21] CG status
// [22] itr
constexpr int kOut = 24;
__global__ void k_collect(const double* __restrict__ dsc, const int* __restrict__ di, const double* __restrict__ ms_its,
                          const int* __restrict__ bar_err, double* __restrict__ out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    out[0] = dsc[DS_FX];
    for (int j = 0; j < 4; j++) out[1 + j] = dsc[DS_GX + j];
    out[5] = dsc[DS_CH];
    out[6] = dsc[DS_RELRES];
    out[7] = dsc[DS_BETA];
    out[8] = dsc[DS_BETA_TMP];
    out[9] = *ms_its;
    out[10] = *bar_err;
    out[11] = di[DI_ITS];
    out[12] = di[DI_STATUS];
    out[13] = di[DI_NAN];
    for (int j = 0; j < 4; j++) {
        out[14 + j] = di[DI_CG_ITS + j];
        out[18 + j] = di[DI_CG_STATUS + j];
    }
    out[22] = di[DI_ITR];
}

// the loop body of main.cpp:72-112 with every stage in its device-driven
// form, in three parts (Ctx::StepGraph)
static int step_part(Ctx& c, int part) {
    const topo_params& p = c.p;
    if (part == 0) {
        k_itr_next<<<1, 32, 0, c.s>>>(c.di.p), note_launch();
        TRET(fem_obj_sens_dev(c, c.XP.p, c.dfdx.p, c.dgdx.p));
        if (p.proj) TRET(projected_sens(c, c.XF.p, c.dfdx.p, c.dgdx.p, p.m, p.x0));
        TRET(filter_sens(c, c.dfdx.p, c.dgdx.p, p.m));
        TRET(mma_movelimit(c, p.Xmin, p.Xmax, p.movlim, c.X.p, c.xmin.p, c.xmax.p));
    } else if (part == 1) {
        TRET(mma_update(c, c.X.p, c.dfdx.p, c.dsc.p + DS_GX, c.dgdx.p, c.xmin.p, c.xmax.p));
        TRET(mma_design_change(c, c.X.p, c.Xold.p, c.dsc.p + DS_CH));
    } else {
        TRET(filter_apply(c, c.X.p, c.XF.p, p.Xmin));
        TRET(heaviside(c, c.XF.p, c.XP.p, p.x0, p.beta0, p.betamax, 0, p.Xmin, p.proj));
        k_collect<<<1, 32, 0, c.s>>>(c.dsc.p, c.di.p, c.mma_scal.p + MS_ITS, c.bar_err.p, c.sg.out.p),
            note_launch();
        TCK(cudaMemcpyAsync(c.hsc.h + 600, c.sg.out.p, kOut * sizeof(double), cudaMemcpyDeviceToHost, c.s));
    }
    TCK(cudaGetLastError());
    return 0;
}

// what the captured graphs depend on: options and the buffers they name
static uint64_t step_sig(const Ctx& c) {
    uint64_t h = 0x5e9ab1e57e9ull;
    const unsigned char* pb = reinterpret_cast<const unsigned char*>(&c.p);
    for (size_t i = 0; i + 8 <= sizeof(c.p); i += 8) {
        uint64_t v;
        std::memcpy(&v, pb + i, 8);
        h = sig_mix(h, v);
    }
    for (const void* q : {(const void*)c.V.p, (const void*)c.Z32.p, (const void*)c.Z64.p, (const void*)c.w.p,
                          (const void*)c.wtmp.p, (const void*)c.red.p, (const void*)c.U.p, (const void*)c.X.p,
                          (const void*)c.XP.p, (const void*)c.Ee64.p, (const void*)c.v32.A0s.p,
                          (const void*)c.v64.A0s.p, (const void*)c.h0.S.p, (const void*)c.mma_scal.p})
        h = sig_mix(h, (uint64_t)(uintptr_t)q);
    h = sig_mix(h, (uint64_t)c.robust_type | (uint64_t)c.constraint_mod << 8);
    const double a[3] = {c.asyminit, c.asymdec, c.asyminc};
    for (double x : a) {
        uint64_t v;
        std::memcpy(&v, &x, 8);
        h = sig_mix(h, v);
    }
    return h;
}

static int capture_part(Ctx& c, int part) {
    Ctx::StepGraph& G = c.sg;
    // the captured work starts after everything queued on the context's stream
    TCK(cudaEventRecord(G.e0, c.s));
    TCK(cudaStreamWaitEvent(G.cap, G.e0, 0));
    cudaStream_t s0 = c.s;
    const bool prof = c.prof.on;
    c.prof.on = false;
    c.s = G.cap;
    c.sg.dd = true;
    c.sg.depth = 0;
    const long l0 = launch_counter();
    cudaError_t e = cudaStreamBeginCapture(G.cap, cudaStreamCaptureModeThreadLocal);
    int rc = e == cudaSuccess ? step_part(c, part) : TOPO_ERR_CUDA;
    // unwind nested captures left open by an error
    while (c.sg.depth > 0) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(c.sg.body[c.sg.depth - 1], &g);
        c.sg.depth--;
    }
    cudaGraph_t g = nullptr;
    if (e == cudaSuccess) e = cudaStreamEndCapture(G.cap, &g);
    c.sg.dd = false;
    c.s = s0;
    c.prof.on = prof;
    const long n = launch_counter() - l0;
    __atomic_fetch_sub(&launch_counter(), n, __ATOMIC_RELAXED);  // nothing ran yet
    cudaGraphExec_t ex = nullptr;
    if (rc >= 0 && e == cudaSuccess && g) e = cudaGraphInstantiate(&ex, g, 0);
    if (g) cudaGraphDestroy(g);
    if (rc < 0 || e != cudaSuccess || !ex) {
        const char* why = e != cudaSuccess ? cudaGetErrorString(e) : last_error();
        cudaGetLastError();
        set_error("step graph capture failed (%s); direct launches from now on", why);
        if (c.p.verbose) fprintf(stderr, "%s\n", last_error());
        return TOPO_ERR_UNSUPPORTED;
    }
    G.exec[part] = ex;
    G.launches[part] = n;
    return 0;
}

static int capture_step(Ctx& c) {
    const auto t0 = std::chrono::steady_clock::now();
    Ctx::StepGraph& G = c.sg;
    if (!G.cap) TCK(cudaStreamCreateWithFlags(&G.cap, cudaStreamNonBlocking));
    for (auto& b : G.body)
        if (!b) TCK(cudaStreamCreateWithFlags(&b, cudaStreamNonBlocking));
    if (!G.e0) {
        TCK(cudaEventCreate(&G.e0));
        TCK(cudaEventCreate(&G.e1));
        TCK(cudaEventCreateWithFlags(&G.p0_done, cudaEventDisableTiming));
    }
    if (!G.out.p) TRET(G.out.alloc(kOut));
    for (int part = 0; part < 3; part++) {
        const int rc = capture_part(c, part);
        if (rc < 0) {
            G.drop();
            G.disabled = true;
            return rc;
        }
    }
    static std::atomic<uint64_t> n_captures{0};
    G.sig = step_sig(c);
    G.gen = ++n_captures;
    G.state_dirty = true;
    c.info.t_capture_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return 0;
}

// ----------------------------------------------------------------- replay
// everything the graphs refer to exists: a direct step of this form (same
// precision) has allocated it and the autotuner has run
static bool graph_ready(const Ctx& c) {
    const bool mixed = c.p.precision == TOPO_PREC_MIXED;
    return c.X.p && c.U.p && c.V.p && c.uku.p && c.L.p && (!tuning_on(c) || c.tune.single_done) &&
           (mixed ? (c.Z32.p && c.v32.allocated) : (c.Z64.p && c.v64.allocated));
}

// Decides whether this step can be replayed (capturing the graphs when
// needed): not the first step of a run (it allocates, autotunes and builds
// the solver state the graphs refer to), not the block solver, not while
// per-kernel timing is on, not after a failed capture.
int opt_step_graph_prepare(Ctx& c, bool* ok) {
    *ok = false;
    Ctx::StepGraph& G = c.sg;
    c.info.step_graph = G.disabled ? -1 : 0;
    // per-kernel event timing (topo_profile_enable) needs the direct launches
    if (G.disabled || c.ncases > 1 || c.itr < 1 || c.prof.on || !graph_ready(c)) return 0;
    if (G.exec[0] && G.sig != step_sig(c)) G.drop();
    if (!G.exec[0] && capture_step(c) < 0) {  // disabled: the caller steps directly
        c.info.step_graph = -1;
        return 0;
    }
    if (G.state_dirty) {
        // the device copies of the host-side loop state (after direct steps)
        c.hsc.h[640] = c.beta_proj;
        c.hsc.h[641] = c.beta_tmp;
        TCK(cudaMemcpyAsync(c.dsc.p + DS_BETA, c.hsc.h + 640, 2 * sizeof(double), cudaMemcpyHostToDevice, c.s));
        int* hi = reinterpret_cast<int*>(c.hsc.h + 642);
        hi[0] = c.itr;
        TCK(cudaMemcpyAsync(c.di.p + DI_ITR, hi, sizeof(int), cudaMemcpyHostToDevice, c.s));
        G.state_dirty = false;
    }
    c.info.step_graph = 1;
    *ok = true;
    return 0;
}

// One event per device, recorded after every replayed part 1 (the MMA update
// with its cooperative dual solve) of any context of this process: the next
// part 1 waits on it, so at most one replayed dual solve runs on a device at a
// time.  With its grid of one block per SM it fits beside the one direct
// dual solve a process runs at a time (mma.cu), whatever the other kernels.
constexpr int kMaxDevices = 64;
static std::mutex& mma_chain_mutex() {
    static std::mutex m;
    return m;
}
static cudaEvent_t mma_chain_event[kMaxDevices];

// launches part p of a prepared step on the context's stream
int opt_step_graph_part(Ctx& c, int part) {
    Ctx::StepGraph& G = c.sg;
    if (part == 1) {
        int dev = 0;
        TCK(cudaGetDevice(&dev));
        if (dev < 0 || dev >= kMaxDevices) {
            set_error("device index %d out of range", dev);
            return TOPO_ERR_UNSUPPORTED;
        }
        std::lock_guard<std::mutex> lk(mma_chain_mutex());
        cudaEvent_t& ev = mma_chain_event[dev];
        if (!ev) TCK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        TCK(cudaStreamWaitEvent(c.s, ev, 0));
        TCK(cudaGraphLaunch(G.exec[1], c.s));
        TCK(cudaEventRecord(ev, c.s));
        __atomic_fetch_add(&launch_counter(), G.launches[1], __ATOMIC_RELAXED);
        return 0;
    }
    if (part == 0) TCK(cudaEventRecord(G.e0, c.s));
    TCK(cudaGraphLaunch(G.exec[part], c.s));
    __atomic_fetch_add(&launch_counter(), G.launches[part], __ATOMIC_RELAXED);
    if (part == 0) TCK(cudaEventRecord(G.p0_done, c.s));
    if (part == 2) {
        TCK(cudaEventRecord(G.e1, c.s));
        c.itr++;
    }
    return 0;
}

// Waits for a launched step and reads its results into the context's info.
int opt_step_graph_finish(Ctx& c) {
    TCK(cudaEventSynchronize(c.sg.e1));
    const double* o = c.hsc.h + 600;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, c.sg.e0, c.sg.e1) != cudaSuccess) { cudaGetLastError(); ms = 0.f; }
    c.info.last_fx = o[0];
    c.info.last_gx0 = o[1];
    c.ch = c.info.last_ch = o[5];
    c.info.fem_relres = o[6];
    c.beta_proj = o[7];
    c.beta_tmp = o[8];
    c.info.mma_inner_its = (int)o[9];
    c.info.fem_its = (int)o[11];
    c.info.fem_status = (int)o[12];
    int cg_status = 0;
    for (int j = 0; j < 4; j++) {
        c.info.filter_its[j] = (int)o[14 + j];
        cg_status = std::max(cg_status, (int)o[18 + j]);
    }
    c.info.t_fem_ms = ms;  // the whole replayed step
    c.info.t_filter_ms = c.info.t_mma_ms = 0.0;
    c.u_valid = true;
    if (c.p.verbose)
        printf("It.: %i, fx: %f, gx[0]: %f, ch.: %f, time: %f\n", c.itr, c.info.last_fx, c.info.last_gx0, c.ch,
               ms * 1e-3);
    if (o[13] != 0.0 || !std::isfinite(c.info.last_fx)) {
        c.u_valid = false;
        amg_reset_warm_start(c);
        set_error("a solve of the design iteration met a non-finite residual");
        return TOPO_ERR_NAN;
    }
    if (o[10] != 0.0) {
        set_error("MMA dual solve: grid barrier timed out");
        return TOPO_ERR_TIMEOUT;
    }
    return (c.info.fem_status || cg_status) ? TOPO_NOT_CONVERGED : 0;
}

// ----------------------------------------------------------------- one graph for a batch of instances
// topo_opt_step_batch with two or more replayable instances launches a single
// graph for all of them.  Each instance's three parts are captured as a branch
// of their own (the branches' kernels overlap on the device), and every
// branch ends with its instance's result copy.  The cooperative dual solves
// (part 1) share one block per SM, as a single replayed part 1 would take:
// with S = min(n, SMs) slots, each instance's grid is capped at SMs / S blocks
// and instance i's part 1 waits for instance i - S's (no waits while n <= SMs).
// The batch graph itself waits on, and records, the per-device part-1 event,
// so no other replayed dual solve runs beside it.  A batch graph is captured
// once per ordered set of instances and kept while none of them recaptures
// its own graphs (StepGraph::gen) or is destroyed.
struct BatchGraph {
    std::vector<Ctx*> ctxs;
    std::vector<uint64_t> gens;
    cudaGraphExec_t exec = nullptr;
    bool failed = false;              // capture failed: these instances use their own graphs
    long launches = 0;                // kernels per replay
    cudaStream_t s = nullptr;         // launch (and capture origin) stream
    cudaEvent_t ev = nullptr;
    std::vector<cudaEvent_t> slot;    // part-1 slots (instances beyond the SM count)
    void drop() {
        if (s) cudaStreamSynchronize(s);
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
    }
    ~BatchGraph() {
        drop();
        if (s) cudaStreamDestroy(s);
        if (ev) cudaEventDestroy(ev);
        for (auto e : slot) cudaEventDestroy(e);
    }
};
constexpr size_t kMaxBatchGraphs = 4;  // sets of instances kept at once (least recently used goes)
static std::mutex& batch_mutex() {
    static std::mutex m;
    return m;
}
// never destroyed: CUDA objects must not be released after the runtime shut down
static std::vector<std::unique_ptr<BatchGraph>>& batch_cache() {
    static auto* v = new std::vector<std::unique_ptr<BatchGraph>>();
    return *v;
}

static int capture_batch(BatchGraph& B) {
    const auto t0 = std::chrono::steady_clock::now();
    if (!B.s) TCK(cudaStreamCreateWithFlags(&B.s, cudaStreamNonBlocking));
    if (!B.ev) TCK(cudaEventCreateWithFlags(&B.ev, cudaEventDisableTiming));
    int dev = 0, nsm = 0;
    TCK(cudaGetDevice(&dev));
    TCK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int n_inst = (int)B.ctxs.size();
    const int n_slot = std::max(1, std::min(n_inst, nsm));
    const int share = std::max(1, nsm / n_slot);  // dual-solve blocks per instance
    while ((int)B.slot.size() < n_slot && n_inst > n_slot) {
        cudaEvent_t e;
        TCK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        B.slot.push_back(e);
    }
    const long l0 = launch_counter();
    int rc = 0;
    cudaError_t e = cudaStreamBeginCapture(B.s, cudaStreamCaptureModeThreadLocal);
    const bool begun = e == cudaSuccess;
    if (begun) e = cudaEventRecord(B.ev, B.s);
    size_t joined = 0;  // branches whose capture stream joined this capture
    for (size_t i = 0; i < B.ctxs.size() && e == cudaSuccess && rc >= 0; i++) {
        Ctx& c = *B.ctxs[i];
        const cudaStream_t s0 = c.s;
        const bool prof = c.prof.on;
        c.prof.on = false;
        c.s = c.sg.cap;
        c.sg.dd = true;
        c.sg.depth = 0;
        c.sg.coop_blocks = share;
        const bool slotted = n_inst > n_slot;
        cudaEvent_t slot_ev = slotted ? B.slot[i % n_slot] : nullptr;
        e = cudaStreamWaitEvent(c.s, B.ev, 0);  // the branch forks off the origin stream
        if (e == cudaSuccess) {
            joined++;
            rc = step_part(c, 0);
            if (rc >= 0 && slotted && (int)i >= n_slot) e = cudaStreamWaitEvent(c.s, slot_ev, 0);
            if (rc >= 0 && e == cudaSuccess) rc = step_part(c, 1);
            if (rc >= 0 && e == cudaSuccess && slotted) e = cudaEventRecord(slot_ev, c.s);
            if (rc >= 0 && e == cudaSuccess) rc = step_part(c, 2);
        }
        while (c.sg.depth > 0) {  // nested captures left open by an error
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(c.sg.body[c.sg.depth - 1], &g);
            c.sg.depth--;
        }
        c.sg.dd = false;
        c.sg.coop_blocks = 0;
        c.s = s0;
        c.prof.on = prof;
    }
    // every branch joins the origin stream again (also after an error, so that
    // the capture ends cleanly)
    for (size_t i = 0; i < joined; i++) {
        const cudaError_t r1 = cudaEventRecord(B.ev, B.ctxs[i]->sg.cap);
        const cudaError_t r2 = cudaStreamWaitEvent(B.s, B.ev, 0);
        if (e == cudaSuccess) e = r1 != cudaSuccess ? r1 : r2;
    }
    cudaGraph_t g = nullptr;
    if (begun) {
        const cudaError_t r = cudaStreamEndCapture(B.s, &g);
        if (e == cudaSuccess) e = r;
    }
    const long n = launch_counter() - l0;
    __atomic_fetch_sub(&launch_counter(), n, __ATOMIC_RELAXED);  // nothing ran yet
    if (rc >= 0 && e == cudaSuccess && g) e = cudaGraphInstantiate(&B.exec, g, 0);
    if (g) cudaGraphDestroy(g);
    if (rc < 0 || e != cudaSuccess || !B.exec) {
        const char* why = e != cudaSuccess ? cudaGetErrorString(e) : last_error();
        cudaGetLastError();
        set_error("batch graph capture failed (%s); the instances' own graphs from now on", why);
        if (B.ctxs[0]->p.verbose) fprintf(stderr, "%s\n", last_error());
        B.exec = nullptr;
        B.failed = true;
        return TOPO_ERR_UNSUPPORTED;
    }
    B.launches = n;
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    for (Ctx* c : B.ctxs) c->info.t_capture_ms = ms;
    return 0;
}

// Launches one iteration of each of the n contexts (every one prepared for
// replay by opt_step_graph_prepare, none in flight) as one graph launch, or
// sets *launched = false when no batch graph can be had (fewer than two
// contexts, a failed capture): the caller then launches the contexts' own
// graphs.  Results are read per context with opt_step_graph_finish.
int opt_step_graph_batch(Ctx* const* cs, int n, bool* launched) {
    *launched = false;
    if (n < 2) return 0;
    std::lock_guard<std::mutex> lk(batch_mutex());
    auto& cache = batch_cache();
    size_t at = cache.size();
    for (size_t k = 0; k < cache.size(); k++)
        if (cache[k]->ctxs.size() == (size_t)n && std::equal(cs, cs + n, cache[k]->ctxs.begin())) at = k;
    if (at == cache.size()) {
        if (cache.size() >= kMaxBatchGraphs) cache.erase(cache.begin());
        auto b = std::make_unique<BatchGraph>();
        b->ctxs.assign(cs, cs + n);
        cache.push_back(std::move(b));
        at = cache.size() - 1;
    } else if (at + 1 != cache.size()) {  // most recently used last
        std::unique_ptr<BatchGraph> b = std::move(cache[at]);
        cache.erase(cache.begin() + at);
        cache.push_back(std::move(b));
        at = cache.size() - 1;
    }
    BatchGraph& B = *cache[at];
    std::vector<uint64_t> gens(n);
    for (int i = 0; i < n; i++) gens[i] = cs[i]->sg.gen;
    if (gens != B.gens) {  // an instance recaptured its graphs: its buffers or options changed
        B.drop();
        B.failed = false;
        B.gens = gens;
    }
    if (B.failed) return 0;
    if (!B.exec && capture_batch(B) < 0) return 0;
    // the graph starts after everything queued on every instance's stream
    for (int i = 0; i < n; i++) {
        TCK(cudaEventRecord(cs[i]->sg.e0, cs[i]->s));
        TCK(cudaStreamWaitEvent(B.s, cs[i]->sg.e0, 0));
    }
    int dev = 0;
    TCK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("device index %d out of range", dev);
        return TOPO_ERR_UNSUPPORTED;
    }
    {
        std::lock_guard<std::mutex> lk2(mma_chain_mutex());
        cudaEvent_t& ev = mma_chain_event[dev];
        if (!ev) TCK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        TCK(cudaStreamWaitEvent(B.s, ev, 0));
        TCK(cudaGraphLaunch(B.exec, B.s));
        TCK(cudaEventRecord(ev, B.s));
    }
    __atomic_fetch_add(&launch_counter(), B.launches, __ATOMIC_RELAXED);
    // each instance's stream continues after the batch
    for (int i = 0; i < n; i++) {
        Ctx& c = *cs[i];
        TCK(cudaEventRecord(c.sg.e1, B.s));
        TCK(cudaStreamWaitEvent(c.s, c.sg.e1, 0));
        c.itr++;
        c.info.step_graph = 2;
    }
    *launched = true;
    return 0;
}

// Drops every batch graph that names context c (it is being destroyed).
void step_batch_forget(const Ctx* c) {
    std::lock_guard<std::mutex> lk(batch_mutex());
    auto& cache = batch_cache();
    for (size_t k = cache.size(); k-- > 0;)
        if (std::find(cache[k]->ctxs.begin(), cache[k]->ctxs.end(), c) != cache[k]->ctxs.end())
            cache.erase(cache.begin() + k);
}

}  // namespace topo
