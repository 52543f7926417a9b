/*
 * topo.h -- C ABI of the B200 (sm_100a) SIMP design-iteration library.
 *
 * One `topo_ctx` is one topology-optimisation job: a device-resident mesh
 * with its SolveFem, PDEFilter and MMA state.  Every entry point replaces one
 * member function of the reference program
 * (gkdas2/Unstructured-FEA-based-Topology-Optimization-in-PETSc-and-Eigen);
 * the replaced interface is cited as file:line beside each declaration.
 *
 * Conventions
 *  - Pointers named *_d are DEVICE pointers (cudaMalloc'd, or from
 *    topo_device_alloc); everything else is host memory.  Ownership never
 *    transfers.  Device vectors over elements have n_elems entries; over
 *    DOFs 3*n_nodes entries, DOF 3n+c = component c of node n
 *    (SolveFem.cpp:38-57).  m constraint vectors are stored back to back.
 *  - Every call returns an int status: TOPO_OK (0); > 0 a usable result with
 *    a warning (TOPO_NOT_CONVERGED: an iterative solve hit its iteration
 *    cap); < 0 an error (nothing to use).  topo_last_error() gives the text.
 *    No C++ exception crosses the ABI.
 *  - All work of one context runs in stream order on the context's stream
 *    (given at creation; NULL = the library creates one).  Calls that
 *    return host scalars synchronise that stream.  One context is not
 *    thread-safe; distinct contexts may be driven from distinct threads.
 */
#ifndef TOPO_H
#define TOPO_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TOPO_OK 0
#define TOPO_NOT_CONVERGED 1
#define TOPO_ERR_ARG (-1)
#define TOPO_ERR_CUDA (-2)
#define TOPO_ERR_OOM (-3)
#define TOPO_ERR_MESH (-4)
#define TOPO_ERR_NAN (-5)
#define TOPO_ERR_UNSUPPORTED (-6)
#define TOPO_ERR_TIMEOUT (-7)
#define TOPO_ERR_IO (-8)
#define TOPO_ERR_CANCELLED (-9)

#define TOPO_PREC_FP64 0  /* FP64 everywhere (the drop-in form) */
#define TOPO_PREC_MIXED 1 /* FP32 AMG V-cycle inside FP64 FGMRES */

typedef struct topo_ctx topo_ctx;

/* Options.  Defaults (topo_params_default) are the reference's:
 * OptPara.cpp:66-78 (Emin 1e-9, Emax 1e6, volfrac 0.12, penal 3, rmin 0.01,
 * Xmin 0.01, Xmax 1, movlim 0.2, x0 0.5, beta0 1, betamax 8, proj off,
 * maxItr 200), SolveFem.cpp:11 (nu 0.3), SolveFem.cpp:126-134 (FGMRES,
 * rtol 1e-5), PDEFilter.cpp:117-120 (CG rtol 1e-5, atol 1e-50, dtol 1e5,
 * maxit 10000), OptPara.cpp:160-177 (MMA a=0, c=1000, d=0, m=1). */
typedef struct topo_params {
    double Emin, Emax, nu, penal, volfrac, rmin, Xmin, Xmax, movlim, x0, beta0, betamax;
    int proj, maxItr, m;
    double ch_tol;         /* main.cpp:70 stop rule `ch > 0.01`; <= 0 disables */
    /* displacement solve: FGMRES + smoothed-aggregation AMG */
    double fem_rtol;
    int fem_restart, fem_maxit;
    int precision;         /* TOPO_PREC_FP64 or TOPO_PREC_MIXED */
    int amg_max_levels;    /* hierarchy depth cap (PCGAMGSetNlevels(pc,4)) */
    int amg_coarse_max;    /* coarsen until a level has <= this many DOFs */
    int amg_smooth_p;      /* 1: smoothed aggregation, 0: plain aggregation */
    int cheb_degree;       /* Chebyshev-Jacobi smoothing steps per sweep */
    int fine_smoother_matfree; /* 1: fine-level smoother uses the element operator */
    /* Helmholtz filter CG (Jacobi) */
    double filter_rtol, filter_atol, filter_dtol;
    int filter_maxit;
    int verbose;           /* 1: print the reference's per-solve lines */
    int amg_rho_its;       /* power iterations for rho(D^-1 A) per level and design iteration */
    double cheb_safety;    /* Chebyshev interval [0.1, 1.1] * cheb_safety * rho */
    int fem_warm_start;    /* 1: start FGMRES from the previous U instead of 0 (the
                              reference zeroes U, SolveFem.cpp:333); same stopping rule */
    int fem_block;         /* n_cases > 1: 1 (default) solves all load cases at once with the
                              block operator and block V-cycle, 0 solves them one by one */
    int fem_graphs;        /* 1 (default): replay each FGMRES Arnoldi step from a CUDA graph
                              captured in an earlier solve with the same buffers */
    int cheb_degree_post;  /* post-smoothing Chebyshev degree (0: same as cheb_degree) */
    int cheb_degree_coarse; /* Chebyshev degree below the finest level (0: as the finest; default 4:
                               the coarse levels are small and latency-bound, and stronger
                               smoothing there cuts FGMRES iterations by about a quarter; 6 cuts
                               them further on one load case but spiked on the 8-case block solve) */
    int autotune;          /* 1 (default): time candidate launch shapes of the hot kernels on
                              this context's own data at its first solve and keep the fastest */
    int amg_coarse_cta;    /* 1: the V-cycle below the first level with <= 8192 DOFs runs in one
                              thread-block cluster (one launch instead of one per sweep); 0 (default):
                              per-sweep kernels, which measured faster at 392k under graph replay */
    int amg_half_fine;     /* mixed form: 1 keeps the level-0 smoother's matrix as FP16
                              D^-1/2 A D^-1/2 (FP32 arithmetic); 0 (default) keeps it FP32 */
    int pdl;               /* 1 (default): V-cycle kernels use programmatic dependent launch (each
                              starts while its predecessor drains and waits on the GPU before it
                              reads the predecessor's output); 0: plain stream order */
    int step_graph;        /* 1: from the second design iteration of a run on, the whole iteration is
                              replayed from CUDA graphs captured once, with the FGMRES and filter-CG
                              loops as conditional graph nodes decided on the device (no host
                              round trip inside an iteration); 0 (default): host-driven iterations.
                              One load case (the block solver always steps directly). */
    int blk_stages;        /* block operator: element-matrix copies in flight per warp, 2 or 3;
                              0 (default): the autotuner times both */
    int deterministic;     /* 1: bitwise-reproducible runs (same inputs, options and GPU give the
                              same bits): the element operators add each node's element
                              contributions in a fixed order (a per-element pass into scratch, then
                              a gather over the node-to-element map) instead of with atomics, no
                              launch shape is autotuned, and several load cases are solved one by
                              one; fixed at creation.  0 (default): atomic scatters (runs agree to
                              rounding) */
} topo_params;

typedef struct topo_solve_info {
    int fem_its;           /* FGMRES iterations of the last displacement solve */
    double fem_relres;     /* ||F - K U|| / ||F|| after it (SolveFem.cpp:142-152) */
    int fem_status;        /* 0 converged, 1 iteration cap */
    int filter_its[4];     /* CG iterations of the last filter solves */
    int amg_levels;
    int amg_dofs[8];       /* DOFs per AMG level */
    int mma_inner_its;     /* dual interior-point steps of the last update */
    double last_fx, last_gx0, last_ch;
    double t_fem_ms, t_filter_ms, t_mma_ms, t_setup_ms; /* stage times (CUDA events) */
    int tuned[4];          /* launch shapes picked by the autotuner: element-operator block,
                              level-0 smoother block, reduction grid, block operator (10 x Ke
                              copies in flight per warp + CTAs per SM, 0: occupancy limit) */
    int tuned_lanes[8];    /* lanes per block row picked for the smoothing and residual products
                              of AMG level l >= 1 (0: not tuned) */
    int step_graph;        /* last design iteration: 1 replayed from the step graph, 2 replayed as
                              a branch of a batch graph (topo_opt_step_batch), 0 stepped
                              directly, -1 the capture failed (direct steps from then on) */
    double t_capture_ms;   /* host time of the last capture of the step graphs (capture and
                              instantiation; 0 before the first); of the whole batch graph when
                              that was captured last */
} topo_solve_info;

/* ---------------------------------------------------------------- basics */
const char* topo_last_error(void);
const char* topo_version(void);
void topo_params_default(topo_params* p);
/* sizeof(topo_params) and sizeof(topo_solve_info) as compiled into the
   library, so a binding (ctypes, cgo, JNI) can check its struct mirrors */
int topo_struct_sizes(size_t* params_bytes, size_t* info_bytes);

/* Device memory for callers without the CUDA runtime. */
int topo_device_alloc(size_t bytes, void** ptr_d);
int topo_device_free(void* ptr_d);
int topo_memcpy_h2d(void* dst_d, const void* src, size_t bytes, topo_ctx* ctx);
int topo_memcpy_d2h(void* dst, const void* src_d, size_t bytes, topo_ctx* ctx);
int topo_sync(topo_ctx* ctx);

/* ---------------------------------------------------------------- mesh + context */
/* Replaces InputMeshData::GetNodeAndElementData + GetBcs
 * (InputMeshData.cpp:33-285) and the SolveFem / PDEFilter / MMA constructors
 * (SolveFem.cpp:6-15, PDEFilter.cpp:7-10,36-140, OptPara.cpp:158-177).
 *   nen          8 (hex8, diagonal numbering) or 4 (tet4)
 *   vertex       n_nodes*3 doubles (vertex.txt rows)
 *   element      n_elems*nen 0-based node ids (element.txt rows)
 *   fixed_dofs   n_fixed DOF ids (fixeddofs.txt)
 *   n_cases      load cases (NUM_LD); case c owns entries
 *                case_ptr[c]..case_ptr[c+1]-1 of load_dofs/load_vals
 *                (loaddof_c.txt / load_c.txt).  n_cases > 1 runs the
 *                block (multi-load) solver; compliance sums over cases.
 *   stream       cudaStream_t for all work of this context, or NULL.
 * Builds the element matrices, volumes (TV), filter operators and the AMG
 * graph hierarchy on the device. */
int topo_create(const topo_params* p, int nen, int n_nodes, const double* vertex, int n_elems,
                const int32_t* element, int n_fixed, const int32_t* fixed_dofs, int n_cases,
                const int32_t* case_ptr, const int32_t* load_dofs, const double* load_vals,
                void* stream, topo_ctx** out);
int topo_destroy(topo_ctx* ctx);
int topo_get_params(topo_ctx* ctx, topo_params* p);
int topo_set_params(topo_ctx* ctx, const topo_params* p);  /* scalar options only */
int topo_sizes(topo_ctx* ctx, int* nen, int* n_nodes, int* n_elems, int* n_cases);
void* topo_stream(topo_ctx* ctx);

/* ---------------------------------------------------------------- SolveFem */
/* Element volumes Vol and their sum TV (SolveFem::ComputeTotalVol,
 * SolveFem.cpp:59-89; 5-tet hex volume SolveFem.cpp:423-467). */
int topo_fem_volumes(topo_ctx* ctx, double* vol_d, double* total_volume);
/* Element stiffness (E = 1) of element e, full ndof_e x ndof_e row-major,
 * DOF order [x0..,y0..,z0..] (SolveFem::Hex8Isoparametric
 * SolveFem.cpp:339-408; tet4/Tet4Isoparametric.cpp:1-41). Host output. */
int topo_fem_element_matrix(topo_ctx* ctx, int e, double* ke);
/* y = K(xphys) u with Dirichlet rows/columns as identity
 * (AssembleFem + MatZeroRowsColumns + MatMult, SolveFem.cpp:267-337). */
int topo_fem_apply(topo_ctx* ctx, const double* xphys_d, const double* u_d, double* y_d);
/* The same for all n_cases load cases at once through the block operator
 * (tensor-core Ke [u_1..u_k] per element): u_d, y_d are [n_cases][3*n_nodes].
 * No counterpart in the reference (its load cases are solved one by one). */
int topo_fem_apply_block(topo_ctx* ctx, const double* xphys_d, const double* u_d, double* y_d);
/* SolveFem::ComputeObjectiveAndSensitivities (SolveFem.h:39-40,
 * SolveFem.cpp:159-265): solves K U = F, then fx = sum E_e u_e'Ke u_e,
 * dfdx, gx[0] = sum x vol / TV - volfrac, dgdx[0] = vol / TV.
 * fx, gx: host; xphys_d, dfdx_d, dgdx_d (m * n_elems): device. */
int topo_fem_obj_sens(topo_ctx* ctx, const double* xphys_d, double* fx, double* gx, double* dfdx_d,
                      double* dgdx_d);
/* The solve alone (SolveFem::ComputeFem, SolveFem.cpp:91-157); U zeroed
 * first, like AssembleFem's VecZeroEntries(U). */
int topo_fem_solve(topo_ctx* ctx, const double* xphys_d, double* u_d);
/* public member U (SolveFem.h:42): last displacement, 3*n_nodes*n_cases */
int topo_fem_displacement(topo_ctx* ctx, double* u_d);
/* von Mises stress per element (stress/ComputeStress.cpp:53-104): centroid
 * stress Emax*D*B*u relaxed by sqrt(x); uses the last displacement. */
int topo_fem_von_mises(topo_ctx* ctx, const double* xphys_d, double* vms_d);

/* No counterpart in the reference.  The compliance and sensitivity reduction
 * of ComputeObjectiveAndSensitivities for a displacement the caller already
 * has, for callers that cannot allocate device memory when they need it
 * (stream-ordered pipelines that must not synchronise the device, hosts that
 * allocate only through their own pool, drivers that forbid allocation after
 * start-up).  It allocates nothing: the caller passes every input and output
 * (device pointers) and the only scratch is a fixed array inside the library
 * (about 130 KB per GPU, held until the process exits).
 *   element_d  n_elems*nen node ids;  ke_d  n_elems * npk packed upper
 *   triangle (row-major, i <= j) of each E = 1 element matrix, npk = 300
 *   (hex8) or 78 (tet4), DOF order [x0..,y0..,z0..];  u_d  3*n_nodes.
 *   Outputs dfdx_d, dgdx_d (n_elems) and fx_gx_d[0] = fx,
 *   fx_gx_d[1] = sum x vol / TV - volfrac, written in stream order.
 * Limit: n_elems <= 1,048,576 (larger meshes are rejected with TOPO_ERR_ARG).
 * The first call on a device looks up the scratch array's device address;
 * make that first call before capturing a stream into a CUDA graph.  All
 * calls share the scratch: calls whose work overlaps on the GPU race. */
int topo_fem_sensitivities_noalloc(int nen, int n_elems, const int32_t* element_d, const double* ke_d,
                                   const double* xphys_d, const double* vol_d, const double* u_d, double Emin,
                                   double Emax, double penal, double total_volume, double volfrac, double* dfdx_d,
                                   double* dgdx_d, double* fx_gx_d, void* stream);

/* ---------------------------------------------------------------- PDEFilter */
/* PDEFilter::Filter (PDEFilter.cpp:142-165): xf = clamp(TFX' KF^-1 TF x, Xmin, 1);
 * the CG warm-starts from the previous solve's RX (PDEFilter.cpp:127). */
int topo_filter_apply(topo_ctx* ctx, const double* x_d, double* xf_d, double Xmin);
/* PDEFilter::ComputeFilteredSens (PDEFilter.cpp:167-183), in place. */
int topo_filter_sens(topo_ctx* ctx, double* dfdx_d, double* dgdx_d, int m);
/* PDEFilter::HeavisideFilter (PDEFilter.cpp:242-293); keeps beta state. */
int topo_heaviside(topo_ctx* ctx, const double* xf_d, double* xp_d, double x0, double beta0,
                   double betamax, int itr, double Xmin, int proj);
/* PDEFilter::ComputeProjectedSens (PDEFilter.cpp:295-341), in place. */
int topo_projected_sens(topo_ctx* ctx, const double* xf_d, double* dfdx_d, double* dgdx_d, int m,
                        double x0);
/* filter warm-start vector RX (n_nodes), read (set=0) or write (set=1) */
int topo_filter_state(topo_ctx* ctx, double* rx_d, int set);

/* ---------------------------------------------------------------- MMA */
/* MMA::SetOuterMovelimit (MMA.h:43, MMA.cpp:370-389) */
int topo_mma_set_outer_movelimit(topo_ctx* ctx, double Xmin, double Xmax, double movlim,
                                 const double* x_d, double* xmin_d, double* xmax_d);
/* MMA::Update (MMA.h:23, MMA.cpp:483-502): GenSub + dual interior point;
 * xval_d updated in place.  gx: host, m values. */
int topo_mma_update(topo_ctx* ctx, double* xval_d, const double* dfdx_d, const double* gx,
                    const double* dgdx_d, const double* xmin_d, const double* xmax_d);
/* MMA::DesignChange (MMA.h:52, MMA.cpp:391-410): ch = max|x - xold|, xold = x */
int topo_mma_design_change(topo_ctx* ctx, const double* x_d, double* xold_d, double* ch);
/* MMA::SetAsymptotes (MMA.h:29, MMA.cpp:345-353) */
int topo_mma_set_asymptotes(topo_ctx* ctx, double init, double decrease, double increase);
/* MMA::SetRobustAsymptotesType (MMA.h:39, MMA.cpp:355-368) */
int topo_mma_set_robust_asymptotes_type(topo_ctx* ctx, int val);
/* MMA::ConstraintModification (MMA.h:32-35) */
int topo_mma_constraint_modification(topo_ctx* ctx, int on);
/* MMA::Restart (MMA.h:26, MMA.cpp:302-342): export xo1, xo2, U, L; and the
 * restart constructor's import (MMA.h:15-18): set=1 loads them with iteration k. */
int topo_mma_restart(topo_ctx* ctx, double* xo1_d, double* xo2_d, double* U_d, double* L_d, int* k,
                     int set);
/* MMA::KKTresidual (MMA.h:47-48, MMA.cpp:412-480) */
int topo_mma_kkt_residual(topo_ctx* ctx, const double* x_d, const double* dfdx_d, const double* gx,
                          const double* dgdx_d, const double* xmin_d, const double* xmax_d,
                          double* norm2, double* norm_inf);

/* ---------------------------------------------------------------- main.cpp loop */
/* Design state owned by the context (OptPara Vecs, OptPara.h:28-52):
 * X = XFiled = XPhys = Xold = volfrac, then the initial Filter +
 * HeavisideFilter of main.cpp:64-66. */
int topo_opt_init(topo_ctx* ctx);
/* One pass of the main.cpp:72-112 loop body.  fx, gx0, ch: host (may be NULL). */
int topo_opt_step(topo_ctx* ctx, int* itr, double* fx, double* gx0, double* ch);
/* Runs the loop `while (itr < maxItr && ch > ch_tol)` (main.cpp:70);
 * hist (host, may be NULL) receives [fx, gx0, ch] per iteration. */
int topo_opt_run(topo_ctx* ctx, int max_itr, double* hist, int* iterations);
/* Advances n independent contexts (design instances) by one design iteration
 * each (no counterpart in the reference, which runs one design per MPI job).
 * Instances whose options select step_graph = 1 and that have done their first
 * iteration are replayed: two or more of them as ONE graph launch in which
 * each instance's iteration is a branch of its own, so their iterations
 * overlap on the device (the cooperative MMA dual solves run one after
 * another).  That batch graph is captured at the first call with a given
 * ordered set of instances and reused while the set and the instances'
 * options and buffers stay the same (the last few sets are kept).  Should its
 * capture fail, every instance's own step graphs are launched on its stream
 * instead.  The other instances step directly, after that launch.
 * status[i] (may be NULL) receives each instance's status, fx[i] (may be NULL)
 * its compliance.  Returns the most severe status: the first error (< 0)
 * met, else the largest warning. */
int topo_opt_step_batch(topo_ctx* const* ctxs, int n, int* status, double* fx);
/* One design iteration without waiting for it (no counterpart in the
 * reference).  With step_graph = 1 and a replayable step, topo_opt_step_async
 * launches the iteration's solve and returns at once; topo_opt_step_query
 * never blocks: it launches the rest of the iteration once the solve has
 * finished, and when the iteration is done sets *done = 1, fills itr, fx, gx0
 * and ch (host, may be NULL) and returns the iteration's status (as
 * topo_opt_step).  Otherwise (the first iteration of a run, the block solver,
 * step_graph = 0) the iteration runs directly inside topo_opt_step_async and
 * the next query reports it.  One host thread can keep many contexts going
 * this way; while an iteration is in flight its context accepts no other
 * optimisation call. */
int topo_opt_step_async(topo_ctx* ctx);
int topo_opt_step_query(topo_ctx* ctx, int* done, int* itr, double* fx, double* gx0, double* ch);
/* Host-buffer form used end to end: uploads the design X (host, n_elems),
 * runs one iteration, downloads the updated X and XPhys (host) and fx. */
int topo_opt_step_host(topo_ctx* ctx, const double* x_in, double* x_out, double* xphys_out, double* fx);
/* access to the context's design vectors; which: 0 X, 1 XPhys, 2 XFiled,
 * 3 Xold, 4 dfdx, 5 dgdx (m*n_elems), 6 xmin, 7 xmax.  Device pointer out. */
int topo_opt_vector(topo_ctx* ctx, int which, double** ptr_d);
int topo_solve_info_get(topo_ctx* ctx, topo_solve_info* info);

/* ---------------------------------------------------------------- serving */
/* Continuous batching of whole optimisation jobs (no counterpart in the
 * reference, which runs one job per MPI launch, main.cpp:35-137): jobs wait
 * in a FIFO until their arrival time, a free slot and their estimated HBM
 * footprint allow admission; each admitted job runs its iterations on its own
 * context and stream, overlapping on the device with the others, and frees
 * its slot and memory when done. */
typedef struct topo_server topo_server;
typedef struct topo_server_stats {
    int jobs_submitted, jobs_done, jobs_failed, max_active;
    long iterations;
    double p50_iter_ms, p99_iter_ms, mean_iter_ms;  /* per design iteration, all jobs */
    double makespan_s, jobs_per_hour, iters_per_s;
    double peak_reserved_bytes;
    double p50_queue_s, p99_queue_s;                /* arrival -> admission */
} topo_server_stats;
/* bytes a job is admitted against (upper estimate of its device footprint) */
size_t topo_estimate_job_bytes(int nen, int n_nodes, int n_elems, int precision);
/* hbm_budget_bytes 0 = 85% of the currently free device memory */
int topo_server_create(size_t hbm_budget_bytes, int max_active, topo_server** out);
int topo_server_destroy(topo_server* s);
/* copies the job's mesh and options; arrival_s is relative to topo_server_run's start */
int topo_server_submit(topo_server* s, const topo_params* p, int nen, int n_nodes, const double* vertex, int n_elems,
                       const int32_t* element, int n_fixed, const int32_t* fixed_dofs, int n_cases,
                       const int32_t* case_ptr, const int32_t* load_dofs, const double* load_vals, int iterations,
                       double arrival_s, int* job_id);
/* Instance batching (no counterpart in the reference): admitted jobs of at
 * most max_elems elements and one load case run their first design iteration
 * on a thread of their own, then join one batch worker that keeps all of them
 * going from one host thread: each job's iterations are replayed from its
 * step graphs (topo_opt_step_async / topo_opt_step_query) and relaunched as
 * soon as they are done.  Batched jobs use the default launch shapes (no
 * autotuning on the shared device).  0 (default) runs every job on its own
 * thread.  Call before topo_server_run. */
int topo_server_set_batching(topo_server* s, int max_elems);
/* runs every submitted job to completion (real-time arrivals); blocks */
int topo_server_run(topo_server* s);
/* Cancels a job; safe to call from another thread while topo_server_run is
 * running.  A queued job is never admitted; a running job stops between two
 * design iterations (none of its work is in flight then) and frees its slot
 * and memory.  Its status becomes TOPO_ERR_CANCELLED and the iterations it
 * finished stay readable through topo_server_job. */
int topo_server_cancel(topo_server* s, int job_id);
/* per-job results (host arrays sized by the caller; NULL to skip):
 * iteration latencies (ms) and compliance history, final XPhys */
int topo_server_job(topo_server* s, int job_id, int* status, int* n_iters, double* iter_ms, double* fx_hist,
                    double* xphys, double* admit_s, double* finish_s);
int topo_server_stats_get(topo_server* s, topo_server_stats* st);

/* Bounds of the device-side waits of this context, for tests of the timeout
 * path (no counterpart in the reference, which has no device waits).
 *   barrier_spins  polls of the MMA dual solve's grid barrier before it gives
 *                  up (0 = default, about a second)
 *   copy_cycles    clock cycles the block operator waits for one bulk copy of
 *                  element matrices (0 = default, about a second)
 *   hold           1: the waits are made to run out without any fault: the
 *                  barrier's last arrival does not release the others and the
 *                  block operator issues no copy.  The call then returns
 *                  TOPO_ERR_TIMEOUT and the context stays usable; 0 restores
 *                  normal operation. */
int topo_test_wait_limits(topo_ctx* ctx, unsigned barrier_spins, unsigned long long copy_cycles, int hold);
/* Test hook (no counterpart in the reference; host only): the order in which
 * the k-load block operator stores the packed upper triangle of an nd x nd
 * element matrix (nd = 24 hex8, 12 tet4) in its shared-memory ring: entry k
 * at perm[k] (nd (nd + 1) / 2 entries).  Returns 1 when the order is free of
 * shared-memory bank conflicts for every half-warp A fragment of the
 * m8n8k4 products, 0 when it fell back to the identity, < 0 on bad
 * arguments. */
int topo_test_block_bank_layout(int nd, int32_t* perm);

/* ---------------------------------------------------------------- instrumentation */
/* Kernel launches issued by this library in this process (all contexts). */
long topo_kernel_launches(void);
/* CUDA-event timing of the hot kernels on the context's stream (no host
 * syncs added): slot 0 element operator K(x)u, 1 level-0 Chebyshev sweep,
 * 2 level-0 residual, 3 Helmholtz-filter operator, 4..7 AMG setup phases
 * (assembly, spectral estimates, Galerkin products, coarse inverse). */
int topo_profile_enable(topo_ctx* ctx, int on);
/* Synchronises, returns launches and summed milliseconds of a slot, resets it. */
int topo_profile_read(topo_ctx* ctx, int slot, long* launches, double* total_ms);
/* AMG hierarchy introspection (replaces what PCGAMG exposes through
 * PCGetCoarseOperators / -pc_gamg_* viewers): after a solve, matrix `which`
 * (0 A_l, 1 P_l, 2 R_l = P_l^T) of level l as plain BSR on the host, blocks
 * row-major.  Call with NULL arrays to get the sizes. */
int topo_amg_level(topo_ctx* ctx, int level, int which, int* nrows, int* ncols, int* bs_r, int* bs_c, long* nnzb,
                   int32_t* rp, int32_t* ci, double* vals);
/* Greedy graph aggregation used for the AMG hierarchy (host only): rows
 * (rp, ci; sorted, self included) of an n-node graph; excl[i] != 0 leaves
 * node i out (-1).  Returns the aggregate count, agg[] the membership. */
int topo_graph_aggregate(int n, const int32_t* rp, const int32_t* ci, const unsigned char* excl, int32_t* agg);

/* ---------------------------------------------------------------- mesh files, output */
/* Synthetic jittered cantilever lattice in the reference's formats (host):
 * nodes (nx+1)(ny+1)(nz+1) with id i + (nx+1)(j + (ny+1)k), splitmix64
 * jitter, hex8 (diagonal numbering) or 6 tet4 per hex.  Pass NULL buffers
 * to query sizes. load_mode 0: unit total -z force on nodes (nx, j, 0);
 * 1: +1 y on nodes (nx, 0, k). */
int topo_gen_cantilever(int nx, int ny, int nz, int nen, double jitter, uint64_t seed, int load_mode,
                        double* vertex, int32_t* element, int32_t* fixed_dofs, int32_t* load_dofs,
                        double* load_vals, int* n_nodes, int* n_elems, int* n_fixed, int* n_loads);
/* k seeded unit point loads on the x = L face (3 DOFs per case). */
int topo_gen_multiload(int nx, int ny, int nz, int k, uint64_t seed, int32_t* load_dofs,
                       double* load_vals);
/* Reads vertex.txt, element.txt, fixeddofs.txt, loaddof_<c>.txt, load_<c>.txt
 * from dir (InputMeshData.cpp:97-149,228-285).  Two passes: NULL buffers
 * query the sizes. */
int topo_read_mesh_dir(const char* dir, int nen, int n_cases, double* vertex, int32_t* element,
                       int32_t* fixed_dofs, int32_t* case_ptr, int32_t* load_dofs, double* load_vals,
                       int* n_nodes, int* n_elems, int* n_fixed, int* n_loads);
/* Write2Vtu::WriteResults (Write2Vtu.cpp:5-174): ASCII .vtu with the
 * diagonal->VTK node reorder, cell type 12 (hex8) / 10 (tet4), point data
 * ux uy uz and cell data xphys, from the context's last U and XPhys.
 * itr 0 -> output_initial.vtu, -1 -> output_final.vtu, else output_<itr>.vtu. */
int topo_write_vtu(topo_ctx* ctx, const char* dir, int itr, const double* xphys_d);
/* (xphys_d: element densities to write, device; NULL = the context's own XPhys) */

#ifdef __cplusplus
}
#endif
#endif
