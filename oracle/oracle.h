/*
 * oracle.h -- CPU restatement of the reference's SIMP design iteration.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this code; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg do, and only as the checker / the timed CPU port.
 *
 * Parity status: the reference (PETSc 3.16.4 + Eigen 3.4 + MPICH) cannot be
 * built in this image, and its mesh blobs are missing, so no output of the
 * reference itself pins this restatement.  It is pinned instead against
 * (a) the element-level known-answer values derived from
 *     SolveFem.cpp:339-408 / PDEFilter.cpp:185-240 (unit cube, tests/golden),
 * (b) the BC fixture counts in mesh/fixeddofs.txt and mesh/loaddof_1.txt,
 * (c) an independent scipy restatement (assembled K + sparse direct solve).
 * Solver iterates (PETSc FGMRES/GAMG/CG) are therefore "parity unpinned":
 * parity is defined against tightly converged FP64 solutions.
 */
#ifndef TOPO_ORACLE_H
#define TOPO_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- mesh generator (jittered lattice, diagonal local numbering) ---- */
void or_gen_lattice_nodes(int nx, int ny, int nz, double h, double jitter,
                          int interior_only, uint64_t seed, double* vertex);
void or_gen_hex8_elements(int nx, int ny, int nz, int* element);
int  or_gen_tet4_elements(int nx, int ny, int nz, const double* vertex, int* element);
int  or_gen_cantilever_bcs(int nx, int ny, int nz, int load_mode,
                           int* fixed_dofs, int* load_dofs, double* load_vals,
                           int* n_fixed, int* n_load);
int  or_gen_multiload(int nx, int ny, int nz, int k, uint64_t seed,
                      int* load_dofs, double* load_vals);

/* ---- element level (SolveFem.cpp / PDEFilter.cpp / tet4) ---- */
void   or_hex8_ke(const double* co /*8x3*/, double nu, double* ke /*24x24*/);
double or_hex8_volume(const double* co /*8x3*/);
void   or_hex8_kehel(const double* co, double rmin, double* ke /*8x8*/, double* T /*8*/);
void   or_tet4_ke(const double* co /*4x3*/, double nu, double* ke /*12x12*/);
double or_tet4_volume(const double* co);
void   or_tet4_kehel(const double* co, double rmin, double* ke /*4x4*/, double* T /*4*/);
void   or_von_mises_hex8(const double* co, double nu, double Emax, double x,
                         const double* ue /*24: x0..x7,y0..y7,z0..z7*/, double* vm);

/* ---- system level ---- */
typedef struct or_params {
    double Emin, Emax, nu, penal, volfrac, rmin, Xmin, Xmax, movlim, x0, beta0, betamax;
    int proj, maxItr, m;
    double fem_rtol; int fem_restart, fem_maxit;
    int precond;         /* 0 = Jacobi, 1 = smoothed-aggregation AMG */
    int amg_levels, amg_coarse_max, cheb_degree, amg_smooth;
    double filter_rtol, filter_atol, filter_dtol; int filter_maxit;
    int nthreads;
} or_params;

typedef struct or_ctx or_ctx;

void    or_params_default(or_params* p);
or_ctx* or_create(const or_params* p, int nen, int nn, const double* vertex, int ne,
                  const int* element, int nfixed, const int* fixed_dofs,
                  int ncases, const int* case_ptr, const int* load_dofs, const double* load_vals);
void    or_destroy(or_ctx* c);

/* SolveFem */
double  or_total_volume(or_ctx* c, double* vol /*ne, may be NULL*/);
void    or_element_ke(or_ctx* c, int e, double* ke /*full ndof_e^2*/);
int     or_assemble(or_ctx* c, const double* xphys);
void    or_get_csr(or_ctx* c, int* n, int* nnz, const int** rp, const int** ci, const double** v);
void    or_get_rhs(or_ctx* c, double* F);
int     or_kmatvec(or_ctx* c, const double* u, double* y);
int     or_solve(or_ctx* c, double* U, int* its, double* relres);
int     or_fem_obj_sens(or_ctx* c, const double* xphys, double* fx, double* gx,
                        double* dfdx, double* dgdx, double* U);
void    or_obj_sens_given_u(or_ctx* c, const double* xphys, const double* U, double* fx, double* gx,
                            double* dfdx, double* dgdx);
/* PDEFilter */
int     or_filter(or_ctx* c, const double* x, double* xf, double Xmin);
int     or_filter_sens(or_ctx* c, double* dfdx, double* dgdx, int m);
void    or_filter_state(or_ctx* c, double* RX, int set);
int     or_filter_last_its(or_ctx* c);
void    or_heaviside(or_ctx* c, const double* xf, double* xp, double x0, double beta0,
                     double betamax, int itr, double Xmin, int proj);
void    or_projected_sens(or_ctx* c, const double* xf, double* dfdx, double* dgdx, int m, double x0);
/* MMA */
void    or_mma_set_outer_movelimit(or_ctx* c, double Xmin, double Xmax, double movlim,
                                   const double* x, double* xmin, double* xmax);
int     or_mma_update(or_ctx* c, double* xval, const double* dfdx, const double* gx,
                      const double* dgdx, const double* xmin, const double* xmax);
double  or_mma_design_change(or_ctx* c, const double* x, double* xold);
void    or_mma_state(or_ctx* c, double* xo1, double* xo2, double* L, double* U, int* k);
void    or_mma_options(or_ctx* c, double asyminit, double asymdec, double asyminc, int robust, int constraint_mod);
void    or_mma_restart_set(or_ctx* c, const double* xo1, const double* xo2, const double* U, const double* L, int k);
void    or_mma_kkt_residual(or_ctx* c, const double* x, const double* dfdx, const double* gx, const double* dgdx,
                            const double* xmin, const double* xmax, double* norm2, double* norm_inf);
/* AMG introspection (aggregation is integer work: compared bit-exactly) */
int     or_amg_aggregates(or_ctx* c, int level, int* agg /*rows of level*/);
/* main.cpp loop: returns iterations done; hist = [fx, gx0, ch] per iteration */
int     or_run(or_ctx* c, int maxItr, double ch_tol, double* hist, double* xphys_out);

#ifdef __cplusplus
}
#endif
#endif
