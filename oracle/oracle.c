/*
 * oracle.c -- CPU restatement (plain C, FP64, OpenMP) of the reference's
 * SIMP design iteration.  TEST INFRASTRUCTURE ONLY: the product library never
 * links or calls it; tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg use it as the checker and as the timed CPU port.
 *
 * Each routine names the reference file:line it restates.  Third-party
 * arithmetic the reference delegates to PETSc 3.16.4 (KSPFGMRES, PCGAMG,
 * KSPCG+PCJACOBI, MatZeroRowsColumns) is restated from PETSc's published
 * algorithms; GAMG is restated as smoothed aggregation (Vanek, Mandel,
 * Brezina 1996) with Chebyshev-Jacobi smoothing, the same algorithm the
 * product runs on the GPU.  Parity of solver iterates is "unpinned" (no
 * reference output exists); parity is defined on tightly converged solves.
 */
#include "oracle.h"
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MAXLEV 8

/* ------------------------------------------------------------------ */
/* splitmix64: the project's seeded jitter source (C, C++ and Python    */
/* produce bit-identical streams).                                      */
/* ------------------------------------------------------------------ */
static uint64_t sm64(uint64_t* s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
static double sm64_unit(uint64_t* s) { return (double)(sm64(s) >> 11) * (1.0 / 9007199254740992.0); }

void or_gen_lattice_nodes(int nx, int ny, int nz, double h, double jitter, int interior_only,
                          uint64_t seed, double* vertex) {
    uint64_t s = seed;
    long n = 0;
    for (int k = 0; k <= nz; k++)
        for (int j = 0; j <= ny; j++)
            for (int i = 0; i <= nx; i++, n++) {
                int idx[3] = {i, j, k}, lim[3] = {nx, ny, nz};
                int interior = (i > 0 && i < nx && j > 0 && j < ny && k > 0 && k < nz);
                for (int c = 0; c < 3; c++) {
                    double u = sm64_unit(&s);
                    double x = (double)idx[c] * h;
                    if (!interior_only || interior) x = x + (2.0 * u - 1.0) * (jitter * h);
                    (void)lim;
                    vertex[3 * n + c] = x;
                }
            }
}

/* diagonal local numbering: local l = a + 2b + 4c -> node (ex+a, ey+b, ez+c)
 * (SolveFem.cpp:352-360 shape-function comment). */
void or_gen_hex8_elements(int nx, int ny, int nz, int* element) {
    long e = 0;
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++, e++)
                for (int l = 0; l < 8; l++) {
                    int a = l & 1, b = (l >> 1) & 1, c = (l >> 2) & 1;
                    element[8 * e + l] = (i + a) + (nx + 1) * ((j + b) + (ny + 1) * (k + c));
                }
}

static double det3(const double* a, const double* b, const double* c) {
    return a[0] * (b[1] * c[2] - b[2] * c[1]) - a[1] * (b[0] * c[2] - b[2] * c[0]) +
           a[2] * (b[0] * c[1] - b[1] * c[0]);
}

/* 6 tets per hex along the 0-7 diagonal (Kuhn split, conforming across
 * hexes); odd permutations get their middle vertices swapped so every tet
 * has positive orientation on the jittered coordinates. */
int or_gen_tet4_elements(int nx, int ny, int nz, const double* vertex, int* element) {
    static const int path[6][2] = {{1, 3}, {1, 5}, {2, 3}, {2, 6}, {4, 5}, {4, 6}};
    int hex[8];
    long e = 0;
    int bad = 0;
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                for (int l = 0; l < 8; l++) {
                    int a = l & 1, b = (l >> 1) & 1, c = (l >> 2) & 1;
                    hex[l] = (i + a) + (nx + 1) * ((j + b) + (ny + 1) * (k + c));
                }
                for (int t = 0; t < 6; t++, e++) {
                    int v[4] = {hex[0], hex[path[t][0]], hex[path[t][1]], hex[7]};
                    double d1[3], d2[3], d3[3];
                    for (int q = 0; q < 3; q++) {
                        d1[q] = vertex[3 * v[1] + q] - vertex[3 * v[0] + q];
                        d2[q] = vertex[3 * v[2] + q] - vertex[3 * v[0] + q];
                        d3[q] = vertex[3 * v[3] + q] - vertex[3 * v[0] + q];
                    }
                    if (det3(d1, d2, d3) < 0.0) { int tmp = v[1]; v[1] = v[2]; v[2] = tmp; }
                    for (int q = 0; q < 4; q++) element[4 * e + q] = v[q];
                    {
                        double e1[3], e2[3], e3[3];
                        for (int q = 0; q < 3; q++) {
                            e1[q] = vertex[3 * v[1] + q] - vertex[3 * v[0] + q];
                            e2[q] = vertex[3 * v[2] + q] - vertex[3 * v[0] + q];
                            e3[q] = vertex[3 * v[3] + q] - vertex[3 * v[0] + q];
                        }
                        if (det3(e1, e2, e3) <= 0.0) bad++;
                    }
                }
            }
    return bad;
}

/* Cantilever BCs selected by lattice index (never by coordinate):
 * fixed = all DOFs of nodes with i = 0 (GetBcs/GetBCs.m:42-51 pattern
 * 3n,3n+1,3n+2); load_mode 0: unit total force in -z spread over nodes with
 * i = nx, k = 0; load_mode 1: +1 in y on each node with i = nx, j = 0 (the
 * orientation of mesh/loaddof_1.txt: 41 DOFs, all 3n+1, value 1). */
int or_gen_cantilever_bcs(int nx, int ny, int nz, int load_mode, int* fixed_dofs, int* load_dofs,
                          double* load_vals, int* n_fixed, int* n_load) {
    int nf = 0, nl = 0;
    for (int k = 0; k <= nz; k++)
        for (int j = 0; j <= ny; j++) {
            int n = 0 + (nx + 1) * (j + (ny + 1) * k);
            if (fixed_dofs) { fixed_dofs[nf] = 3 * n; fixed_dofs[nf + 1] = 3 * n + 1; fixed_dofs[nf + 2] = 3 * n + 2; }
            nf += 3;
        }
    if (load_mode == 0) {
        for (int j = 0; j <= ny; j++) {
            int n = nx + (nx + 1) * (j + (ny + 1) * 0);
            if (load_dofs) { load_dofs[nl] = 3 * n + 2; load_vals[nl] = -1.0 / (double)(ny + 1); }
            nl++;
        }
    } else {
        for (int k = 0; k <= nz; k++) {
            int n = nx + (nx + 1) * (0 + (ny + 1) * k);
            if (load_dofs) { load_dofs[nl] = 3 * n + 1; load_vals[nl] = 1.0; }
            nl++;
        }
    }
    *n_fixed = nf;
    *n_load = nl;
    return 0;
}

/* k point loads at seeded random nodes of the x = L face, random unit
 * directions; case c owns load_dofs/vals[3c..3c+2]. */
int or_gen_multiload(int nx, int ny, int nz, int k, uint64_t seed, int* load_dofs, double* load_vals) {
    uint64_t s = seed;
    for (int c = 0; c < k; c++) {
        int j = (int)(sm64_unit(&s) * (double)(ny + 1));
        int kk = (int)(sm64_unit(&s) * (double)(nz + 1));
        if (j > ny) j = ny;
        if (kk > nz) kk = nz;
        double zc = 2.0 * sm64_unit(&s) - 1.0;
        double ph = 6.283185307179586 * sm64_unit(&s);
        double rr = sqrt(1.0 - zc * zc);
        double d[3] = {rr * cos(ph), rr * sin(ph), zc};
        int n = nx + (nx + 1) * (j + (ny + 1) * kk);
        for (int q = 0; q < 3; q++) { load_dofs[3 * c + q] = 3 * n + q; load_vals[3 * c + q] = d[q]; }
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* element level                                                        */
/* ------------------------------------------------------------------ */
static double inv3(const double J[9], double Ji[9]) {
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

static void elastic_D(double nu, double D[36]) {
    /* SolveFem.cpp:370-376 (E = 1) */
    double lam = nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    double mu = 1.0 / (2.0 * (1.0 + nu));
    memset(D, 0, 36 * sizeof(double));
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) D[6 * a + b] = lam + (a == b ? 2.0 * mu : 0.0);
    D[21] = mu; D[28] = mu; D[35] = mu;
}

/* strain-displacement B (6 x 3n), DOF order [x0..xn-1, y.., z..]
 * (SolveFem.cpp:400 B layout, rows exx eyy ezz gxy gyz gxz). */
static void build_B(int nn, const double* dN /*3 x nn*/, double* B /*6 x 3nn*/) {
    int nd = 3 * nn;
    memset(B, 0, 6 * nd * sizeof(double));
    for (int l = 0; l < nn; l++) {
        double dx = dN[l], dy = dN[nn + l], dz = dN[2 * nn + l];
        B[0 * nd + l] = dx;
        B[1 * nd + nn + l] = dy;
        B[2 * nd + 2 * nn + l] = dz;
        B[3 * nd + l] = dy; B[3 * nd + nn + l] = dx;
        B[4 * nd + nn + l] = dz; B[4 * nd + 2 * nn + l] = dy;
        B[5 * nd + l] = dz; B[5 * nd + 2 * nn + l] = dx;
    }
}

static void add_BtDB(int nd, const double* B, const double* D, double s, double* ke) {
    double DB[6 * 24];
    for (int a = 0; a < 6; a++)
        for (int j = 0; j < nd; j++) {
            double t = 0.0;
            for (int b = 0; b < 6; b++) t += D[6 * a + b] * B[b * nd + j];
            DB[a * nd + j] = t;
        }
    for (int i = 0; i < nd; i++)
        for (int j = 0; j < nd; j++) {
            double t = 0.0;
            for (int a = 0; a < 6; a++) t += B[a * nd + i] * DB[a * nd + j];
            ke[i * nd + j] += s * t;
        }
}

/* rounded 3-point Gauss rule (SolveFem.cpp:364-365, PDEFilter.cpp:195-196) */
static const double GP[3] = {-0.775, 0.0, 0.775};
static const double GW[3] = {0.556, 0.889, 0.556};

/* derivatives of the diagonal-numbering trilinear shape functions
 * (SolveFem.cpp:390-395, row(0)=d/dxi, row(1)=d/deta, row(2)=d/dzeta) */
static void hex8_dN(double xi, double eta, double zeta, double* Nd /*3x8*/) {
    for (int l = 0; l < 8; l++) {
        double sa = (l & 1) ? 1.0 : -1.0, sb = (l & 2) ? 1.0 : -1.0, sc = (l & 4) ? 1.0 : -1.0;
        Nd[l] = 0.125 * sa * (1.0 + sb * eta) * (1.0 + sc * zeta);
        Nd[8 + l] = 0.125 * sb * (1.0 + sa * xi) * (1.0 + sc * zeta);
        Nd[16 + l] = 0.125 * sc * (1.0 + sa * xi) * (1.0 + sb * eta);
    }
}

/* SolveFem::Hex8Isoparametric (SolveFem.cpp:339-408) */
void or_hex8_ke(const double* co, double nu, double* ke) {
    double D[36], Nd[24], J[9], Ji[9], dN[24], B[6 * 24];
    elastic_D(nu, D);
    memset(ke, 0, 576 * sizeof(double));
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            for (int k = 0; k < 3; k++) {
                hex8_dN(GP[i], GP[j], GP[k], Nd);
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++) {
                        double t = 0.0;
                        for (int l = 0; l < 8; l++) t += Nd[8 * a + l] * co[3 * l + b];
                        J[3 * a + b] = t;
                    }
                double det = inv3(J, Ji);
                for (int a = 0; a < 3; a++)
                    for (int l = 0; l < 8; l++)
                        dN[8 * a + l] = Ji[3 * a] * Nd[l] + Ji[3 * a + 1] * Nd[8 + l] + Ji[3 * a + 2] * Nd[16 + l];
                build_B(8, dN, B);
                add_BtDB(24, B, D, GW[i] * GW[j] * GW[k] * det, ke);
            }
}

/* SolveFem::ComputeVolOfHex (SolveFem.cpp:423-467): 5 tets, |.| summed */
double or_hex8_volume(const double* co) {
#define SUBV(o, a, b) double o[3] = {co[3 * (a)] - co[3 * (b)], co[3 * (a) + 1] - co[3 * (b) + 1], co[3 * (a) + 2] - co[3 * (b) + 2]}
    SUBV(s61, 5, 0); SUBV(s62, 5, 1); SUBV(s64, 5, 3);
    double p1 = 1.0 / 6.0 * det3(s61, s62, s64);
    SUBV(s71, 6, 0); SUBV(s74, 6, 3); SUBV(s73, 6, 2);
    double p2 = 1.0 / 6.0 * det3(s71, s74, s73);
    SUBV(o16, 0, 5); SUBV(o15, 0, 4); SUBV(o17, 0, 6);
    double p3 = 1.0 / 6.0 * det3(o16, o15, o17);
    SUBV(f46, 3, 5); SUBV(f47, 3, 6); SUBV(f48, 3, 7);
    double p4 = 1.0 / 6.0 * det3(f46, f47, f48);
    SUBV(s67, 5, 6);
    double p5 = 1.0 / 6.0 * det3(s61, s64, s67);
#undef SUBV
    return fabs(p1) + fabs(p2) + fabs(p3) + fabs(p4) + fabs(p5);
}

/* PDEFilter::KeHel (PDEFilter.cpp:185-240) */
void or_hex8_kehel(const double* co, double rmin, double* ke, double* T) {
    double r = 1.0 / (2.0 * sqrt(3.0)) * rmin;
    double r2 = r * r;
    memset(ke, 0, 64 * sizeof(double));
    memset(T, 0, 8 * sizeof(double));
    double Nd[24], N[8], J[9], Ji[9], Dn[24];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            for (int k = 0; k < 3; k++) {
                double s = GP[i], t = GP[j], v = GP[k];
                for (int l = 0; l < 8; l++) {
                    double sa = (l & 1) ? 1.0 : -1.0, sb = (l & 2) ? 1.0 : -1.0, sc = (l & 4) ? 1.0 : -1.0;
                    N[l] = (1.0 + sa * s) * (1.0 + sb * t) * (1.0 + sc * v) * 0.125;
                }
                hex8_dN(s, t, v, Nd);
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++) {
                        double q = 0.0;
                        for (int l = 0; l < 8; l++) q += Nd[8 * a + l] * co[3 * l + b];
                        J[3 * a + b] = q;
                    }
                double det = inv3(J, Ji);
                for (int a = 0; a < 3; a++)
                    for (int l = 0; l < 8; l++)
                        Dn[8 * a + l] = Ji[3 * a] * Nd[l] + Ji[3 * a + 1] * Nd[8 + l] + Ji[3 * a + 2] * Nd[16 + l];
                double w = GW[i] * GW[j] * GW[k];
                for (int p = 0; p < 8; p++) {
                    for (int q = 0; q < 8; q++) {
                        double g = Dn[p] * Dn[q] + Dn[8 + p] * Dn[8 + q] + Dn[16 + p] * Dn[16 + q];
                        ke[8 * p + q] += w * (r2 * g + N[p] * N[q]) * det;
                    }
                    T[p] += w * N[p] * det;
                }
            }
}

static void tet4_J(const double* co, double J[9]) {
    /* Ndiff = [-1 1 0 0; -1 0 1 0; -1 0 0 1] (tet4/Tet4Isoparametric.cpp:27-29) */
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) J[3 * a + b] = co[3 * (a + 1) + b] - co[b];
}

/* SolveFem::Tet4Isoparametric (tet4/Tet4Isoparametric.cpp:1-41) */
void or_tet4_ke(const double* co, double nu, double* ke) {
    double D[36], J[9], Ji[9], dN[12], B[6 * 12];
    static const double Nd[12] = {-1, 1, 0, 0, -1, 0, 1, 0, -1, 0, 0, 1};
    elastic_D(nu, D);
    tet4_J(co, J);
    double det = inv3(J, Ji);
    double detJ = sqrt(det * det); /* sqrt(det(J J^T)) */
    for (int a = 0; a < 3; a++)
        for (int l = 0; l < 4; l++)
            dN[4 * a + l] = Ji[3 * a] * Nd[l] + Ji[3 * a + 1] * Nd[4 + l] + Ji[3 * a + 2] * Nd[8 + l];
    build_B(4, dN, B);
    memset(ke, 0, 144 * sizeof(double));
    add_BtDB(12, B, D, 1.0 / 6.0 * detJ, ke);
}

/* tet volume (the reference leaves the tet4 volume routine to the user) */
double or_tet4_volume(const double* co) {
    double J[9];
    tet4_J(co, J);
    return fabs(det3(J, J + 3, J + 6)) / 6.0;
}

/* PDEFilter::KeHel, tet4 variant (tet4/KeHel.cpp:1-47): 4-point Hammer rule */
void or_tet4_kehel(const double* co, double rmin, double* ke, double* T) {
    double r = 1.0 / (2.0 * sqrt(3.0)) * rmin;
    double r2 = r * r;
    double a = (5.0 + 3.0 * sqrt(5.0)) / 20.0, b = (5.0 - sqrt(5.0)) / 20.0;
    double G[4][3] = {{a, b, b}, {b, a, b}, {b, b, a}, {b, b, b}};
    static const double Nd[12] = {-1, 1, 0, 0, -1, 0, 1, 0, -1, 0, 0, 1};
    double J[9], Ji[9], Dn[12];
    tet4_J(co, J);
    double det = inv3(J, Ji);
    for (int aa = 0; aa < 3; aa++)
        for (int l = 0; l < 4; l++)
            Dn[4 * aa + l] = Ji[3 * aa] * Nd[l] + Ji[3 * aa + 1] * Nd[4 + l] + Ji[3 * aa + 2] * Nd[8 + l];
    memset(ke, 0, 16 * sizeof(double));
    memset(T, 0, 4 * sizeof(double));
    for (int g = 0; g < 4; g++) {
        double s = G[g][0], t = G[g][1], v = G[g][2];
        double N[4] = {1 - s - t - v, s, t, v};
        for (int p = 0; p < 4; p++) {
            for (int q = 0; q < 4; q++) {
                double gg = Dn[p] * Dn[q] + Dn[4 + p] * Dn[4 + q] + Dn[8 + p] * Dn[8 + q];
                ke[4 * p + q] += 1.0 / 24.0 * (r2 * gg + N[p] * N[q]) * det;
            }
            T[p] += 1.0 / 24.0 * N[p] * det;
        }
    }
}

/* SolveFem::ComputeStress (stress/ComputeStress.cpp:53-104): centroid stress,
 * relaxed by sqrt(x), von Mises. ue in [x0..x7, y0..y7, z0..z7] order. */
void or_von_mises_hex8(const double* co, double nu, double Emax, double x, const double* ue, double* vm) {
    double D[36], Nd[24], J[9], Ji[9], dN[24], B[6 * 24];
    elastic_D(nu, D);
    hex8_dN(0.0, 0.0, 0.0, Nd);
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
            double t = 0.0;
            for (int l = 0; l < 8; l++) t += Nd[8 * a + l] * co[3 * l + b];
            J[3 * a + b] = t;
        }
    inv3(J, Ji);
    for (int a = 0; a < 3; a++)
        for (int l = 0; l < 8; l++)
            dN[8 * a + l] = Ji[3 * a] * Nd[l] + Ji[3 * a + 1] * Nd[8 + l] + Ji[3 * a + 2] * Nd[16 + l];
    build_B(8, dN, B);
    double eps[6], es[6];
    for (int a = 0; a < 6; a++) {
        double t = 0.0;
        for (int j = 0; j < 24; j++) t += B[a * 24 + j] * ue[j];
        eps[a] = t;
    }
    double sr = sqrt(x);
    for (int a = 0; a < 6; a++) {
        double t = 0.0;
        for (int b = 0; b < 6; b++) t += D[6 * a + b] * eps[b];
        es[a] = sr * (Emax * t);
    }
    *vm = (1.0 / sqrt(2.0)) * sqrt((es[0] - es[1]) * (es[0] - es[1]) + (es[0] - es[2]) * (es[0] - es[2]) +
                                   (es[1] - es[2]) * (es[1] - es[2]) +
                                   6.0 * (es[3] * es[3] + es[4] * es[4] + es[5] * es[5]));
}

/* ------------------------------------------------------------------ */
/* sparse helpers (scalar CSR)                                          */
/* ------------------------------------------------------------------ */
typedef struct { int n, m; int* rp; int* ci; double* v; } csr;

static void csr_free(csr* a) { free(a->rp); free(a->ci); free(a->v); memset(a, 0, sizeof(*a)); }

static void spmv(const csr* a, const double* x, double* y) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < a->n; i++) {
        double t = 0.0;
        for (int p = a->rp[i]; p < a->rp[i + 1]; p++) t += a->v[p] * x[a->ci[p]];
        y[i] = t;
    }
}

static int cmp_int(const void* a, const void* b) { int x = *(const int*)a, y = *(const int*)b; return (x > y) - (x < y); }

static csr csr_transpose(const csr* a) {
    csr t; t.n = a->m; t.m = a->n;
    t.rp = calloc(t.n + 1, sizeof(int));
    int nnz = a->rp[a->n];
    t.ci = malloc((nnz ? nnz : 1) * sizeof(int));
    t.v = malloc((nnz ? nnz : 1) * sizeof(double));
    for (int p = 0; p < nnz; p++) t.rp[a->ci[p] + 1]++;
    for (int i = 0; i < t.n; i++) t.rp[i + 1] += t.rp[i];
    int* pos = malloc((t.n + 1) * sizeof(int));
    memcpy(pos, t.rp, (t.n + 1) * sizeof(int));
    for (int i = 0; i < a->n; i++)
        for (int p = a->rp[i]; p < a->rp[i + 1]; p++) {
            int q = pos[a->ci[p]]++;
            t.ci[q] = i; t.v[q] = a->v[p];
        }
    free(pos);
    return t;
}

/* Gustavson C = A*B; rows sorted; structural entries kept */
static csr spgemm(const csr* A, const csr* B) {
    csr C; C.n = A->n; C.m = B->m;
    C.rp = calloc(C.n + 1, sizeof(int));
    int nt = 1;
#ifdef _OPENMP
    nt = omp_get_max_threads();
#endif
    int** marks = malloc(nt * sizeof(int*));
    for (int t = 0; t < nt; t++) { marks[t] = malloc(B->m * sizeof(int)); for (int j = 0; j < B->m; j++) marks[t][j] = -1; }
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < A->n; i++) {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        int* mk = marks[tid];
        int cnt = 0;
        for (int p = A->rp[i]; p < A->rp[i + 1]; p++) {
            int k = A->ci[p];
            for (int q = B->rp[k]; q < B->rp[k + 1]; q++) {
                int j = B->ci[q];
                if (mk[j] != i) { mk[j] = i; cnt++; }
            }
        }
        C.rp[i + 1] = cnt;
    }
    for (int i = 0; i < C.n; i++) C.rp[i + 1] += C.rp[i];
    int nnz = C.rp[C.n];
    C.ci = malloc((nnz ? nnz : 1) * sizeof(int));
    C.v = malloc((nnz ? nnz : 1) * sizeof(double));
    for (int t = 0; t < nt; t++) for (int j = 0; j < B->m; j++) marks[t][j] = -1;
    double** acc = malloc(nt * sizeof(double*));
    for (int t = 0; t < nt; t++) acc[t] = calloc(B->m, sizeof(double));
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < A->n; i++) {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        int* mk = marks[tid];
        double* ac = acc[tid];
        int base = C.rp[i], cnt = 0;
        for (int p = A->rp[i]; p < A->rp[i + 1]; p++) {
            int k = A->ci[p];
            double av = A->v[p];
            for (int q = B->rp[k]; q < B->rp[k + 1]; q++) {
                int j = B->ci[q];
                if (mk[j] != i) { mk[j] = i; C.ci[base + cnt++] = j; ac[j] = 0.0; }
                ac[j] += av * B->v[q];
            }
        }
        qsort(C.ci + base, cnt, sizeof(int), cmp_int);
        for (int q = 0; q < cnt; q++) C.v[base + q] = ac[C.ci[base + q]];
    }
    for (int t = 0; t < nt; t++) { free(marks[t]); free(acc[t]); }
    free(marks); free(acc);
    return C;
}

static double dot(int n, const double* a, const double* b) {
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (int i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}

/* ------------------------------------------------------------------ */
/* context                                                              */
/* ------------------------------------------------------------------ */
typedef struct {
    csr A, P, R;
    double* dinv;
    double rho;
    int bs, nnode;        /* block size and node count of this level */
    int* agg;             /* node -> aggregate (level nodes), -1 none */
    int nagg;
    double *r, *x, *b, *t, *d;
    /* coarsest dense LU */
    double* lu; int* piv;
} level_t;

struct or_ctx {
    or_params p;
    int nen, ndof_e, nn, ne, n;
    double* vertex;
    int* elem;
    int *n2e_ptr, *n2e;
    int *adj_ptr, *adj;
    unsigned short* bpos;
    double* ke;          /* ne * ndof_e^2 (full) */
    double* vol;
    double TV;
    int nfixed;
    int* fixed;
    unsigned char* isfixed;
    double* F;
    double* Ee;
    csr K;
    /* filter */
    double* kf;          /* ne * nen^2 */
    double* tf;          /* ne * nen */
    csr KF;
    double* fdiag;
    double *RX, *TX, *fr, *fz, *fp, *fw;
    int filter_its;
    double beta_proj, beta_tmp;
    /* solver */
    int solve_its;
    double solve_relres;
    level_t lev[MAXLEV];
    int nlev;
    int amg_built;
    /* MMA (MMA.cpp) */
    int mk;
    double asyminit, asymdec, asyminc;
    int constraintModification, RobustAsymptotesType;
    double *a, *c, *d, *y, *lam, *mu, *s, *b, *grad, *Hess;
    double z;
    double *L, *U, *alpha, *beta, *p0, *q0, *pij, *qij, *xo1, *xo2;
};

void or_params_default(or_params* p) {
    /* OptPara.cpp:66-78 defaults, SolveFem.cpp:11 nu, SolveFem.cpp:134
     * FGMRES rtol, PDEFilter.cpp:117-120 CG tolerances */
    p->Emin = 1.0e-9; p->Emax = 1.0e6; p->nu = 0.3; p->penal = 3.0; p->volfrac = 0.12;
    p->rmin = 0.01; p->Xmin = 0.01; p->Xmax = 1.0; p->movlim = 0.2; p->x0 = 0.5;
    p->beta0 = 1.0; p->betamax = 8.0; p->proj = 0; p->maxItr = 200; p->m = 1;
    p->fem_rtol = 1.0e-5; p->fem_restart = 30; p->fem_maxit = 10000;
    p->precond = 1; p->amg_levels = 4; p->amg_coarse_max = 2000; p->cheb_degree = 2; p->amg_smooth = 1;
    p->filter_rtol = 1.0e-5; p->filter_atol = 1.0e-50; p->filter_dtol = 1.0e5; p->filter_maxit = 10000;
    p->nthreads = 0;
}

static void build_graph(or_ctx* c) {
    int nn = c->nn, ne = c->ne, nen = c->nen;
    c->n2e_ptr = calloc(nn + 1, sizeof(int));
    for (long q = 0; q < (long)ne * nen; q++) c->n2e_ptr[c->elem[q] + 1]++;
    for (int i = 0; i < nn; i++) c->n2e_ptr[i + 1] += c->n2e_ptr[i];
    c->n2e = malloc((size_t)ne * nen * sizeof(int));
    int* pos = malloc((nn + 1) * sizeof(int));
    memcpy(pos, c->n2e_ptr, (nn + 1) * sizeof(int));
    for (long q = 0; q < (long)ne * nen; q++) c->n2e[pos[c->elem[q]]++] = (int)q;
    free(pos);
    /* adjacency incl. self, sorted */
    c->adj_ptr = calloc(nn + 1, sizeof(int));
    int* mark = malloc(nn * sizeof(int));
    for (int i = 0; i < nn; i++) mark[i] = -1;
    for (int i = 0; i < nn; i++) {
        int cnt = 0;
        for (int p = c->n2e_ptr[i]; p < c->n2e_ptr[i + 1]; p++) {
            int e = c->n2e[p] / nen;
            for (int l = 0; l < nen; l++) { int j = c->elem[e * nen + l]; if (mark[j] != i) { mark[j] = i; cnt++; } }
        }
        c->adj_ptr[i + 1] = cnt;
    }
    for (int i = 0; i < nn; i++) c->adj_ptr[i + 1] += c->adj_ptr[i];
    c->adj = malloc(c->adj_ptr[nn] * sizeof(int));
    for (int i = 0; i < nn; i++) mark[i] = -1;
    for (int i = 0; i < nn; i++) {
        int cnt = 0, base = c->adj_ptr[i];
        for (int p = c->n2e_ptr[i]; p < c->n2e_ptr[i + 1]; p++) {
            int e = c->n2e[p] / nen;
            for (int l = 0; l < nen; l++) { int j = c->elem[e * nen + l]; if (mark[j] != i) { mark[j] = i; c->adj[base + cnt++] = j; } }
        }
        qsort(c->adj + base, cnt, sizeof(int), cmp_int);
    }
    free(mark);
    c->bpos = malloc((size_t)ne * nen * nen * sizeof(unsigned short));
#pragma omp parallel for schedule(static)
    for (int e = 0; e < ne; e++)
        for (int p = 0; p < nen; p++) {
            int np = c->elem[e * nen + p];
            for (int q = 0; q < nen; q++) {
                int nq = c->elem[e * nen + q];
                int lo = c->adj_ptr[np], hi = c->adj_ptr[np + 1] - 1;
                while (lo < hi) { int mid = (lo + hi) / 2; if (c->adj[mid] < nq) lo = mid + 1; else hi = mid; }
                c->bpos[((size_t)e * nen + p) * nen + q] = (unsigned short)(lo - c->adj_ptr[np]);
            }
        }
    /* scalar CSR pattern of K: row 3n+c has columns 3m+d for m in adj(n) */
    int n = 3 * nn;
    c->n = n;
    c->K.n = c->K.m = n;
    c->K.rp = malloc((n + 1) * sizeof(int));
    c->K.rp[0] = 0;
    for (int i = 0; i < nn; i++) {
        int deg = c->adj_ptr[i + 1] - c->adj_ptr[i];
        for (int cc = 0; cc < 3; cc++) c->K.rp[3 * i + cc + 1] = c->K.rp[3 * i + cc] + 3 * deg;
    }
    int nnz = c->K.rp[n];
    c->K.ci = malloc(nnz * sizeof(int));
    c->K.v = calloc(nnz, sizeof(double));
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nn; i++)
        for (int cc = 0; cc < 3; cc++) {
            int base = c->K.rp[3 * i + cc], q = 0;
            for (int p = c->adj_ptr[i]; p < c->adj_ptr[i + 1]; p++)
                for (int d = 0; d < 3; d++) c->K.ci[base + q++] = 3 * c->adj[p] + d;
        }
}

or_ctx* or_create(const or_params* p, int nen, int nn, const double* vertex, int ne, const int* element,
                  int nfixed, const int* fixed_dofs, int ncases, const int* case_ptr, const int* load_dofs,
                  const double* load_vals) {
    if (nen != 8 && nen != 4) return NULL;
    or_ctx* c = calloc(1, sizeof(or_ctx));
    c->p = *p;
#ifdef _OPENMP
    if (p->nthreads > 0) omp_set_num_threads(p->nthreads);
#endif
    c->nen = nen; c->ndof_e = 3 * nen; c->nn = nn; c->ne = ne;
    c->vertex = malloc((size_t)nn * 3 * sizeof(double));
    memcpy(c->vertex, vertex, (size_t)nn * 3 * sizeof(double));
    c->elem = malloc((size_t)ne * nen * sizeof(int));
    memcpy(c->elem, element, (size_t)ne * nen * sizeof(int));
    for (long q = 0; q < (long)ne * nen; q++)
        if (c->elem[q] < 0 || c->elem[q] >= nn) { free(c->vertex); free(c->elem); free(c); return NULL; }
    build_graph(c);
    int nd = c->ndof_e;
    c->ke = malloc((size_t)ne * nd * nd * sizeof(double));
    c->vol = malloc(ne * sizeof(double));
    c->kf = malloc((size_t)ne * nen * nen * sizeof(double));
    c->tf = malloc((size_t)ne * nen * sizeof(double));
    double TV = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : TV)
    for (int e = 0; e < ne; e++) {
        double co[24];
        for (int l = 0; l < nen; l++)
            for (int q = 0; q < 3; q++) co[3 * l + q] = c->vertex[3 * c->elem[e * nen + l] + q];
        if (nen == 8) {
            or_hex8_ke(co, p->nu, c->ke + (size_t)e * 576);
            c->vol[e] = or_hex8_volume(co);
            or_hex8_kehel(co, p->rmin, c->kf + (size_t)e * 64, c->tf + (size_t)e * 8);
        } else {
            or_tet4_ke(co, p->nu, c->ke + (size_t)e * 144);
            c->vol[e] = or_tet4_volume(co);
            or_tet4_kehel(co, p->rmin, c->kf + (size_t)e * 16, c->tf + (size_t)e * 4);
        }
        TV += c->vol[e];
    }
    c->TV = TV;
    /* BCs */
    int n = c->n;
    c->nfixed = nfixed;
    c->fixed = malloc((nfixed ? nfixed : 1) * sizeof(int));
    memcpy(c->fixed, fixed_dofs, nfixed * sizeof(int));
    c->isfixed = calloc(n, 1);
    for (int i = 0; i < nfixed; i++) if (fixed_dofs[i] >= 0 && fixed_dofs[i] < n) c->isfixed[fixed_dofs[i]] = 1;
    c->F = calloc((size_t)n * (ncases > 0 ? ncases : 1), sizeof(double));
    /* AssembleFem (SolveFem.cpp:277-282): VecSetValues INSERT of each case
     * into the same F.  The oracle keeps one column per case; ncases == 1
     * reproduces the reference. */
    for (int k = 0; k < ncases; k++)
        for (int q = case_ptr[k]; q < case_ptr[k + 1]; q++) c->F[(size_t)k * n + load_dofs[q]] = load_vals[q];
    for (int k = 0; k < ncases; k++)
        for (int i = 0; i < nfixed; i++) c->F[(size_t)k * n + fixed_dofs[i]] = 0.0;
    c->Ee = malloc(ne * sizeof(double));
    /* filter KF (CSR on the node graph), diag */
    c->KF.n = c->KF.m = nn;
    c->KF.rp = malloc((nn + 1) * sizeof(int));
    memcpy(c->KF.rp, c->adj_ptr, (nn + 1) * sizeof(int));
    c->KF.ci = malloc(c->adj_ptr[nn] * sizeof(int));
    memcpy(c->KF.ci, c->adj, c->adj_ptr[nn] * sizeof(int));
    c->KF.v = calloc(c->adj_ptr[nn], sizeof(double));
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nn; i++)
        for (int q = c->n2e_ptr[i]; q < c->n2e_ptr[i + 1]; q++) {
            int e = c->n2e[q] / nen, l = c->n2e[q] % nen;
            for (int m = 0; m < nen; m++)
                c->KF.v[c->adj_ptr[i] + c->bpos[((size_t)e * nen + l) * nen + m]] += c->kf[((size_t)e * nen + l) * nen + m];
        }
    c->fdiag = malloc(nn * sizeof(double));
    for (int i = 0; i < nn; i++)
        for (int q = c->KF.rp[i]; q < c->KF.rp[i + 1]; q++) if (c->KF.ci[q] == i) c->fdiag[i] = c->KF.v[q];
    c->RX = calloc(nn, sizeof(double));
    c->TX = calloc(nn, sizeof(double));
    c->fr = calloc(nn, sizeof(double)); c->fz = calloc(nn, sizeof(double));
    c->fp = calloc(nn, sizeof(double)); c->fw = calloc(nn, sizeof(double));
    /* MMA (MMA.cpp:178-224; OptPara.cpp:158-177 a=0, c=1000, d=0) */
    int m = p->m;
    c->asyminit = 0.5; c->asymdec = 0.7; c->asyminc = 1.2;
    c->a = calloc(m, sizeof(double)); c->c = calloc(m, sizeof(double)); c->d = calloc(m, sizeof(double));
    for (int j = 0; j < m; j++) c->c[j] = 1000.0;
    c->y = calloc(m, sizeof(double)); c->lam = calloc(m, sizeof(double)); c->mu = calloc(m, sizeof(double));
    c->s = calloc(2 * m, sizeof(double)); c->b = calloc(m, sizeof(double)); c->grad = calloc(m, sizeof(double));
    c->Hess = calloc(m * m, sizeof(double));
    c->L = calloc(ne, sizeof(double)); c->U = calloc(ne, sizeof(double));
    c->alpha = calloc(ne, sizeof(double)); c->beta = calloc(ne, sizeof(double));
    c->p0 = calloc(ne, sizeof(double)); c->q0 = calloc(ne, sizeof(double));
    c->pij = calloc((size_t)ne * m, sizeof(double)); c->qij = calloc((size_t)ne * m, sizeof(double));
    c->xo1 = calloc(ne, sizeof(double)); c->xo2 = calloc(ne, sizeof(double));
    return c;
}

static void level_free(level_t* L) {
    csr_free(&L->A); csr_free(&L->P); csr_free(&L->R);
    free(L->dinv); free(L->agg); free(L->r); free(L->x); free(L->b); free(L->t); free(L->d);
    free(L->lu); free(L->piv);
    memset(L, 0, sizeof(*L));
}

void or_destroy(or_ctx* c) {
    if (!c) return;
    for (int l = 0; l < MAXLEV; l++) {
        if (l == 0) { c->lev[0].A.rp = NULL; c->lev[0].A.ci = NULL; c->lev[0].A.v = NULL; }
        level_free(&c->lev[l]);
    }
    free(c->vertex); free(c->elem); free(c->n2e_ptr); free(c->n2e); free(c->adj_ptr); free(c->adj);
    free(c->bpos); free(c->ke); free(c->vol); free(c->fixed); free(c->isfixed); free(c->F); free(c->Ee);
    csr_free(&c->K); free(c->kf); free(c->tf); csr_free(&c->KF); free(c->fdiag);
    free(c->RX); free(c->TX); free(c->fr); free(c->fz); free(c->fp); free(c->fw);
    free(c->a); free(c->c); free(c->d); free(c->y); free(c->lam); free(c->mu); free(c->s); free(c->b);
    free(c->grad); free(c->Hess); free(c->L); free(c->U); free(c->alpha); free(c->beta); free(c->p0);
    free(c->q0); free(c->pij); free(c->qij); free(c->xo1); free(c->xo2);
    free(c);
}

double or_total_volume(or_ctx* c, double* vol) {
    if (vol) memcpy(vol, c->vol, c->ne * sizeof(double));
    return c->TV;
}

void or_element_ke(or_ctx* c, int e, double* ke) {
    int nd = c->ndof_e;
    memcpy(ke, c->ke + (size_t)e * nd * nd, nd * nd * sizeof(double));
}

/* SolveFem::AssembleFem (SolveFem.cpp:267-337): K = sum_e E(rho_e) Ke_e,
 * E = Emin + rho^p (Emax - Emin) (:304), then MatZeroRowsColumns(diag 1). */
int or_assemble(or_ctx* c, const double* xphys) {
    const or_params* p = &c->p;
    int nen = c->nen, nd = c->ndof_e;
#pragma omp parallel for schedule(static)
    for (int e = 0; e < c->ne; e++) c->Ee[e] = p->Emin + pow(xphys[e], p->penal) * (p->Emax - p->Emin);
    memset(c->K.v, 0, c->K.rp[c->n] * sizeof(double));
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < c->nn; i++) {
        int deg = c->adj_ptr[i + 1] - c->adj_ptr[i];
        for (int q = c->n2e_ptr[i]; q < c->n2e_ptr[i + 1]; q++) {
            int e = c->n2e[q] / nen, l = c->n2e[q] % nen;
            const double* ke = c->ke + (size_t)e * nd * nd;
            double E = c->Ee[e];
            for (int cc = 0; cc < 3; cc++) {
                int row = 3 * i + cc;
                double* rv = c->K.v + c->K.rp[row];
                const double* kr = ke + (cc * nen + l) * nd;
                for (int m = 0; m < nen; m++) {
                    int slot = c->bpos[((size_t)e * nen + l) * nen + m];
                    for (int d = 0; d < 3; d++) rv[3 * slot + d] += E * kr[d * nen + m];
                }
            }
        }
        (void)deg;
    }
    /* Dirichlet: zero rows and columns, unit diagonal */
#pragma omp parallel for schedule(static)
    for (int r = 0; r < c->n; r++) {
        int fr = c->isfixed[r];
        for (int q = c->K.rp[r]; q < c->K.rp[r + 1]; q++) {
            int col = c->K.ci[q];
            if (fr || c->isfixed[col]) c->K.v[q] = (fr && col == r) ? 1.0 : 0.0;
        }
    }
    c->amg_built = 0;
    return 0;
}

void or_get_csr(or_ctx* c, int* n, int* nnz, const int** rp, const int** ci, const double** v) {
    *n = c->n; *nnz = c->K.rp[c->n]; *rp = c->K.rp; *ci = c->K.ci; *v = c->K.v;
}

void or_get_rhs(or_ctx* c, double* F) { memcpy(F, c->F, c->n * sizeof(double)); }

int or_kmatvec(or_ctx* c, const double* u, double* y) { spmv(&c->K, u, y); return 0; }

/* ------------------------------------------------------------------ */
/* smoothed-aggregation AMG (restatement of PCGAMG's algorithm family) */
/* ------------------------------------------------------------------ */

/* Greedy aggregation on a node graph: phase 1 roots a new aggregate at each
 * node whose (non-excluded) neighbourhood is untouched; phase 2 attaches the
 * remaining nodes to the phase-1 aggregate of their first aggregated
 * neighbour; phase 3 makes singletons of anything left. */
static int aggregate(int nn, const int* rp, const int* ci, const unsigned char* excl, int* agg) {
    int na = 0;
    for (int i = 0; i < nn; i++) agg[i] = excl && excl[i] ? -2 : -1;
    for (int i = 0; i < nn; i++) {
        if (agg[i] != -1) continue;
        int ok = 1;
        for (int p = rp[i]; p < rp[i + 1]; p++) { int j = ci[p]; if (j != i && agg[j] >= 0) { ok = 0; break; } }
        if (!ok) continue;
        for (int p = rp[i]; p < rp[i + 1]; p++) { int j = ci[p]; if (agg[j] == -1) agg[j] = na; }
        agg[i] = na;
        na++;
    }
    int* a1 = malloc(nn * sizeof(int));
    memcpy(a1, agg, nn * sizeof(int));
    for (int i = 0; i < nn; i++) {
        if (a1[i] != -1) continue;
        for (int p = rp[i]; p < rp[i + 1]; p++) { int j = ci[p]; if (a1[j] >= 0) { agg[i] = a1[j]; break; } }
    }
    free(a1);
    for (int i = 0; i < nn; i++) if (agg[i] == -1) agg[i] = na++;
    return na;
}

/* power iteration on D^-1 A (10 steps, deterministic start) */
static double est_rho(const csr* A, const double* dinv, double* v, double* w) {
    int n = A->n;
    for (int i = 0; i < n; i++) v[i] = 1.0 + 0.1 * (double)((i * 7919) % 13) / 13.0;
    double lam = 0.0;
    for (int it = 0; it < 10; it++) {
        double nv = sqrt(dot(n, v, v));
        for (int i = 0; i < n; i++) v[i] /= nv;
        spmv(A, v, w);
        for (int i = 0; i < n; i++) w[i] *= dinv[i];
        lam = dot(n, v, w);
        memcpy(v, w, n * sizeof(double));
    }
    return lam;
}

static void dense_lu(int n, double* a, int* piv) {
    for (int k = 0; k < n; k++) {
        int pr = k; double mx = fabs(a[k * n + k]);
        for (int i = k + 1; i < n; i++) if (fabs(a[i * n + k]) > mx) { mx = fabs(a[i * n + k]); pr = i; }
        piv[k] = pr;
        if (pr != k) for (int j = 0; j < n; j++) { double t = a[k * n + j]; a[k * n + j] = a[pr * n + j]; a[pr * n + j] = t; }
        double d = a[k * n + k];
        if (d == 0.0) { a[k * n + k] = d = 1.0; }
        for (int i = k + 1; i < n; i++) {
            double f = a[i * n + k] / d;
            a[i * n + k] = f;
            for (int j = k + 1; j < n; j++) a[i * n + j] -= f * a[k * n + j];
        }
    }
}
static void dense_lu_solve(int n, const double* a, const int* piv, double* x) {
    for (int k = 0; k < n; k++) if (piv[k] != k) { double t = x[k]; x[k] = x[piv[k]]; x[piv[k]] = t; }
    for (int i = 0; i < n; i++) { double s = x[i]; for (int j = 0; j < i; j++) s -= a[i * n + j] * x[j]; x[i] = s; }
    for (int i = n - 1; i >= 0; i--) { double s = x[i]; for (int j = i + 1; j < n; j++) s -= a[i * n + j] * x[j]; x[i] = s / a[i * n + i]; }
}

static void level_alloc_vecs(level_t* L) {
    int n = L->A.n;
    L->r = calloc(n, sizeof(double)); L->x = calloc(n, sizeof(double)); L->b = calloc(n, sizeof(double));
    L->t = calloc(n, sizeof(double)); L->d = calloc(n, sizeof(double));
    L->dinv = malloc(n * sizeof(double));
    for (int i = 0; i < n; i++) {
        double dg = 0.0;
        for (int q = L->A.rp[i]; q < L->A.rp[i + 1]; q++) if (L->A.ci[q] == i) dg = L->A.v[q];
        L->dinv[i] = dg != 0.0 ? 1.0 / dg : 1.0;
    }
}

static int amg_setup(or_ctx* c) {
    const or_params* p = &c->p;
    for (int l = 1; l < MAXLEV; l++) level_free(&c->lev[l]);
    { level_t* L0 = &c->lev[0]; free(L0->dinv); free(L0->agg); free(L0->r); free(L0->x); free(L0->b); free(L0->t); free(L0->d);
      csr_free(&L0->P); csr_free(&L0->R); free(L0->lu); free(L0->piv); memset(L0, 0, sizeof(*L0)); }
    level_t* L = &c->lev[0];
    L->A = c->K;   /* borrowed */
    L->bs = 3; L->nnode = c->nn;
    level_alloc_vecs(L);
    /* level-0 graph = mesh node graph; nodes with all DOFs fixed excluded */
    int* grp = c->adj_ptr; int* gci = c->adj;
    int* own_rp = NULL; int* own_ci = NULL;
    unsigned char* excl = calloc(c->nn, 1);
    for (int i = 0; i < c->nn; i++) excl[i] = c->isfixed[3 * i] && c->isfixed[3 * i + 1] && c->isfixed[3 * i + 2];
    /* near null space B (n x 6): rigid body modes */
    int nlev = 1;
    double* B = NULL;
    int lvl = 0;
    while (1) {
        L = &c->lev[lvl];
        int n = L->A.n, bs = L->bs, nnode = L->nnode;
        if (lvl + 1 >= p->amg_levels || n <= p->amg_coarse_max || lvl + 1 >= MAXLEV) break;
        L->agg = malloc(nnode * sizeof(int));
        int na = aggregate(nnode, grp, gci, lvl == 0 ? excl : NULL, L->agg);
        L->nagg = na;
        if (na == 0 || na >= nnode) { break; }
        /* tentative prolongator per aggregate by modified Gram-Schmidt */
        int nc = 6 * na;
        int* cnt = calloc(na + 1, sizeof(int));
        for (int i = 0; i < nnode; i++) if (L->agg[i] >= 0) cnt[L->agg[i] + 1]++;
        for (int a = 0; a < na; a++) cnt[a + 1] += cnt[a];
        int* mem = malloc((cnt[na] ? cnt[na] : 1) * sizeof(int));
        int* fill = malloc((na + 1) * sizeof(int));
        memcpy(fill, cnt, (na + 1) * sizeof(int));
        for (int i = 0; i < nnode; i++) if (L->agg[i] >= 0) mem[fill[L->agg[i]]++] = i;
        free(fill);
        double* Bn = calloc((size_t)nc * 6, sizeof(double));
        csr Pt; Pt.n = n; Pt.m = nc; Pt.rp = calloc(n + 1, sizeof(int));
        for (int i = 0; i < nnode; i++)
            for (int q = 0; q < bs; q++) {
                int row = bs * i + q;
                int free_row = (lvl > 0) || !c->isfixed[row];
                Pt.rp[row + 1] = (L->agg[i] >= 0 && free_row) ? 6 : 0;
            }
        for (int r = 0; r < n; r++) Pt.rp[r + 1] += Pt.rp[r];
        Pt.ci = malloc((Pt.rp[n] ? Pt.rp[n] : 1) * sizeof(int));
        Pt.v = malloc((Pt.rp[n] ? Pt.rp[n] : 1) * sizeof(double));
#pragma omp parallel for schedule(dynamic, 16)
        for (int a = 0; a < na; a++) {
            int m0 = cnt[a], m1 = cnt[a + 1];
            int rows = 0;
            for (int t = m0; t < m1; t++) for (int q = 0; q < bs; q++) { int row = bs * mem[t] + q; if (lvl > 0 || !c->isfixed[row]) rows++; }
            double* Q = calloc((size_t)(rows ? rows : 1) * 6, sizeof(double));
            int* rid = malloc((rows ? rows : 1) * sizeof(int));
            double cen[3] = {0, 0, 0};
            if (lvl == 0) {
                for (int t = m0; t < m1; t++) for (int q = 0; q < 3; q++) cen[q] += c->vertex[3 * mem[t] + q];
                for (int q = 0; q < 3; q++) cen[q] /= (double)(m1 - m0);
            }
            int rr = 0;
            for (int t = m0; t < m1; t++) {
                int i = mem[t];
                for (int q = 0; q < bs; q++) {
                    int row = bs * i + q;
                    if (lvl == 0 && c->isfixed[row]) continue;
                    rid[rr] = row;
                    if (lvl == 0) {
                        double x = c->vertex[3 * i] - cen[0], y = c->vertex[3 * i + 1] - cen[1], z = c->vertex[3 * i + 2] - cen[2];
                        double rb[3][6] = {{1, 0, 0, -y, 0, z}, {0, 1, 0, x, -z, 0}, {0, 0, 1, 0, y, -x}};
                        for (int j = 0; j < 6; j++) Q[rr * 6 + j] = rb[q][j];
                    } else {
                        for (int j = 0; j < 6; j++) Q[rr * 6 + j] = B[(size_t)row * 6 + j];
                    }
                    rr++;
                }
            }
            double Rm[36] = {0};
            for (int j = 0; j < 6; j++) {
                double n0 = 0.0;
                for (int r2 = 0; r2 < rows; r2++) n0 += Q[r2 * 6 + j] * Q[r2 * 6 + j];
                n0 = sqrt(n0);
                for (int i2 = 0; i2 < j; i2++) {
                    double h = 0.0;
                    for (int r2 = 0; r2 < rows; r2++) h += Q[r2 * 6 + i2] * Q[r2 * 6 + j];
                    Rm[i2 * 6 + j] = h;
                    for (int r2 = 0; r2 < rows; r2++) Q[r2 * 6 + j] -= h * Q[r2 * 6 + i2];
                }
                double nr = 0.0;
                for (int r2 = 0; r2 < rows; r2++) nr += Q[r2 * 6 + j] * Q[r2 * 6 + j];
                nr = sqrt(nr);
                if (nr <= 1e-10 * n0 || nr == 0.0) {
                    for (int r2 = 0; r2 < rows; r2++) Q[r2 * 6 + j] = 0.0;
                    Rm[j * 6 + j] = 0.0;
                } else {
                    for (int r2 = 0; r2 < rows; r2++) Q[r2 * 6 + j] /= nr;
                    Rm[j * 6 + j] = nr;
                }
            }
            for (int r2 = 0; r2 < rows; r2++) {
                int row = rid[r2];
                int base = Pt.rp[row];
                for (int j = 0; j < 6; j++) { Pt.ci[base + j] = 6 * a + j; Pt.v[base + j] = Q[r2 * 6 + j]; }
            }
            for (int i2 = 0; i2 < 6; i2++) for (int j = 0; j < 6; j++) Bn[(size_t)(6 * a + i2) * 6 + j] = Rm[i2 * 6 + j];
            free(Q); free(rid);
        }
        free(cnt); free(mem);
        /* smoothing P = (I - w D^-1 A) Pt, w = 4 / (3 rho) */
        L->rho = est_rho(&L->A, L->dinv, L->t, L->d);
        if (p->amg_smooth) {
            csr AP = spgemm(&L->A, &Pt);
            double w = 4.0 / (3.0 * L->rho);
            /* P = Pt - w Dinv AP on the union pattern (AP's pattern contains Pt's
             * since A has a full diagonal) */
            L->P = AP;
            for (int r = 0; r < n; r++) {
                int q0 = Pt.rp[r];
                for (int q = L->P.rp[r]; q < L->P.rp[r + 1]; q++) {
                    double v = -w * L->dinv[r] * L->P.v[q];
                    for (int t = Pt.rp[r]; t < Pt.rp[r + 1]; t++) if (Pt.ci[t] == L->P.ci[q]) v += Pt.v[t];
                    L->P.v[q] = v;
                }
                (void)q0;
            }
            csr_free(&Pt);
        } else {
            L->P = Pt;
        }
        L->R = csr_transpose(&L->P);
        csr APm = spgemm(&L->A, &L->P);
        level_t* Lc = &c->lev[lvl + 1];
        Lc->A = spgemm(&L->R, &APm);
        csr_free(&APm);
        Lc->bs = 6; Lc->nnode = na;
        /* zero diagonal (degenerate mode) -> unit */
        for (int i = 0; i < Lc->A.n; i++) {
            int has = 0;
            for (int q = Lc->A.rp[i]; q < Lc->A.rp[i + 1]; q++) if (Lc->A.ci[q] == i && Lc->A.v[q] != 0.0) has = 1;
            if (!has) for (int q = Lc->A.rp[i]; q < Lc->A.rp[i + 1]; q++) if (Lc->A.ci[q] == i) Lc->A.v[q] = 1.0;
        }
        level_alloc_vecs(Lc);
        /* coarse node graph from the block pattern */
        free(own_rp); free(own_ci);
        own_rp = calloc(na + 1, sizeof(int));
        int* mk = malloc(na * sizeof(int));
        for (int a = 0; a < na; a++) mk[a] = -1;
        int tot = 0;
        for (int a = 0; a < na; a++) {
            for (int rr2 = 0; rr2 < 6; rr2++) {
                int row = 6 * a + rr2;
                for (int q = Lc->A.rp[row]; q < Lc->A.rp[row + 1]; q++) { int b2 = Lc->A.ci[q] / 6; if (mk[b2] != a) { mk[b2] = a; tot++; } }
            }
            own_rp[a + 1] = tot;
        }
        own_ci = malloc((tot ? tot : 1) * sizeof(int));
        for (int a = 0; a < na; a++) mk[a] = -1;
        for (int a = 0; a < na; a++) {
            int base = own_rp[a], k2 = 0;
            for (int rr2 = 0; rr2 < 6; rr2++) {
                int row = 6 * a + rr2;
                for (int q = Lc->A.rp[row]; q < Lc->A.rp[row + 1]; q++) { int b2 = Lc->A.ci[q] / 6; if (mk[b2] != a) { mk[b2] = a; own_ci[base + k2++] = b2; } }
            }
            qsort(own_ci + base, k2, sizeof(int), cmp_int);
        }
        free(mk);
        grp = own_rp; gci = own_ci;
        free(B);
        B = Bn;
        lvl++;
        nlev = lvl + 1;
    }
    free(B); free(excl); free(own_rp); free(own_ci);
    /* coarsest: dense LU */
    level_t* Lc = &c->lev[nlev - 1];
    int nc = Lc->A.n;
    Lc->lu = calloc((size_t)nc * nc, sizeof(double));
    Lc->piv = malloc(nc * sizeof(int));
    for (int i = 0; i < nc; i++)
        for (int q = Lc->A.rp[i]; q < Lc->A.rp[i + 1]; q++) Lc->lu[(size_t)i * nc + Lc->A.ci[q]] = Lc->A.v[q];
    dense_lu(nc, Lc->lu, Lc->piv);
    for (int l = 0; l < nlev - 1; l++) if (c->lev[l].rho == 0.0) c->lev[l].rho = est_rho(&c->lev[l].A, c->lev[l].dinv, c->lev[l].t, c->lev[l].d);
    c->nlev = nlev;
    c->amg_built = 1;
    return 0;
}

/* Chebyshev(k) with Jacobi on [0.1, 1.1] * rho */
static void cheby(level_t* L, const double* b, double* x, int deg, int zero_init) {
    int n = L->A.n;
    double emax = 1.1 * L->rho, emin = 0.1 * L->rho;
    double theta = 0.5 * (emax + emin), delta = 0.5 * (emax - emin);
    double sigma = theta / delta, rho = 1.0 / sigma;
    double* r = L->r; double* d = L->d;
    if (zero_init) { memcpy(r, b, n * sizeof(double)); memset(x, 0, n * sizeof(double)); }
    else { spmv(&L->A, x, r); for (int i = 0; i < n; i++) r[i] = b[i] - r[i]; }
    for (int i = 0; i < n; i++) { d[i] = L->dinv[i] * r[i] / theta; x[i] += d[i]; }
    for (int k = 1; k < deg; k++) {
        spmv(&L->A, d, L->t);
        for (int i = 0; i < n; i++) r[i] -= L->t[i];
        double rn = 1.0 / (2.0 * sigma - rho);
        for (int i = 0; i < n; i++) { d[i] = rn * rho * d[i] + 2.0 * rn / delta * L->dinv[i] * r[i]; x[i] += d[i]; }
        rho = rn;
    }
}

static void vcycle(or_ctx* c, int l, const double* b, double* x) {
    level_t* L = &c->lev[l];
    int n = L->A.n;
    if (l == c->nlev - 1) {
        memcpy(x, b, n * sizeof(double));
        dense_lu_solve(n, L->lu, L->piv, x);
        return;
    }
    int deg = c->p.cheb_degree;
    cheby(L, b, x, deg, 1);
    spmv(&L->A, x, L->t);
    for (int i = 0; i < n; i++) L->t[i] = b[i] - L->t[i];
    level_t* Lc = &c->lev[l + 1];
    spmv(&L->R, L->t, Lc->b);
    vcycle(c, l + 1, Lc->b, Lc->x);
    spmv(&L->P, Lc->x, L->t);
    for (int i = 0; i < n; i++) x[i] += L->t[i];
    cheby(L, b, x, deg, 0);
}

static void precond(or_ctx* c, const double* v, double* z) {
    if (c->p.precond == 0) {
        for (int i = 0; i < c->n; i++) {
            double dg = 1.0;
            for (int q = c->K.rp[i]; q < c->K.rp[i + 1]; q++) if (c->K.ci[q] == i) dg = c->K.v[q];
            z[i] = v[i] / dg;
        }
        return;
    }
    vcycle(c, 0, v, z);
}

/* FGMRES(restart), right preconditioned, classical Gram-Schmidt,
 * converged when |g_{j+1}| <= max(rtol*||b||, 1e-50) (PETSc KSPFGMRES +
 * KSPConvergedDefault with a nonzero initial guess; SolveFem.cpp:124-139). */
static int fgmres(or_ctx* c, const double* b, double* x, double rtol, int restart, int maxit, int* its_out, double* res_out) {
    int n = c->n;
    double* V = malloc((size_t)(restart + 1) * n * sizeof(double));
    double* Z = malloc((size_t)restart * n * sizeof(double));
    double* w = malloc(n * sizeof(double));
    double* H = calloc((size_t)(restart + 1) * restart, sizeof(double));
    double* cs = calloc(restart, sizeof(double));
    double* sn = calloc(restart, sizeof(double));
    double* g = calloc(restart + 1, sizeof(double));
    double* yv = calloc(restart, sizeof(double));
    double bnorm = sqrt(dot(n, b, b));
    double ttol = rtol * bnorm > 1e-50 ? rtol * bnorm : 1e-50;
    int its = 0, conv = 0;
    double res = 0.0;
    while (!conv && its < maxit) {
        spmv(&c->K, x, w);
        for (int i = 0; i < n; i++) V[i] = b[i] - w[i];
        double beta = sqrt(dot(n, V, V));
        res = beta;
        if (beta <= ttol) { conv = 1; break; }
        for (int i = 0; i < n; i++) V[i] /= beta;
        memset(g, 0, (restart + 1) * sizeof(double));
        g[0] = beta;
        int j;
        int kdone = 0;
        for (j = 0; j < restart && its < maxit; j++) {
            double* vj = V + (size_t)j * n;
            double* zj = Z + (size_t)j * n;
            precond(c, vj, zj);
            spmv(&c->K, zj, w);
            for (int i = 0; i <= j; i++) H[i * restart + j] = dot(n, w, V + (size_t)i * n);
            for (int i = 0; i <= j; i++) {
                double h = H[i * restart + j];
                double* vi = V + (size_t)i * n;
#pragma omp parallel for schedule(static)
                for (int q = 0; q < n; q++) w[q] -= h * vi[q];
            }
            double hn = sqrt(dot(n, w, w));
            H[(j + 1) * restart + j] = hn;
            for (int i = 0; i < j; i++) {
                double t1 = H[i * restart + j], t2 = H[(i + 1) * restart + j];
                H[i * restart + j] = cs[i] * t1 + sn[i] * t2;
                H[(i + 1) * restart + j] = -sn[i] * t1 + cs[i] * t2;
            }
            double hjj = H[j * restart + j], hj1 = H[(j + 1) * restart + j];
            double den = sqrt(hjj * hjj + hj1 * hj1);
            if (den == 0.0) { cs[j] = 1.0; sn[j] = 0.0; } else { cs[j] = hjj / den; sn[j] = hj1 / den; }
            H[j * restart + j] = cs[j] * hjj + sn[j] * hj1;
            H[(j + 1) * restart + j] = 0.0;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            its++;
            res = fabs(g[j + 1]);
            kdone = j + 1;
            if (res <= ttol || hn == 0.0) { conv = res <= ttol; break; }
            double* vn = V + (size_t)(j + 1) * n;
            for (int q = 0; q < n; q++) vn[q] = w[q] / hn;
        }
        /* x += Z y */
        for (int i = kdone - 1; i >= 0; i--) {
            double s = g[i];
            for (int k = i + 1; k < kdone; k++) s -= H[i * restart + k] * yv[k];
            yv[i] = s / H[i * restart + i];
        }
        for (int k = 0; k < kdone; k++) {
            double* zk = Z + (size_t)k * n;
#pragma omp parallel for schedule(static)
            for (int q = 0; q < n; q++) x[q] += yv[k] * zk[q];
        }
    }
    free(V); free(Z); free(w); free(H); free(cs); free(sn); free(g); free(yv);
    *its_out = its;
    *res_out = res;
    return conv ? 0 : 1;
}

/* SolveFem::ComputeFem (SolveFem.cpp:91-157): U zeroed, FGMRES + AMG. */
int or_solve(or_ctx* c, double* U, int* its, double* relres) {
    int n = c->n;
    memset(U, 0, n * sizeof(double));
    if (c->p.precond == 1 && !c->amg_built) amg_setup(c);
    int rc = fgmres(c, c->F, U, c->p.fem_rtol, c->p.fem_restart, c->p.fem_maxit, &c->solve_its, &c->solve_relres);
    /* true residual ||F - K U|| / ||F|| (SolveFem.cpp:142-152) */
    double* w = malloc(n * sizeof(double));
    spmv(&c->K, U, w);
    for (int i = 0; i < n; i++) w[i] = c->F[i] - w[i];
    double rn = sqrt(dot(n, w, w)), fn = sqrt(dot(n, c->F, c->F));
    free(w);
    c->solve_relres = fn > 0 ? rn / fn : rn;
    if (its) *its = c->solve_its;
    if (relres) *relres = c->solve_relres;
    return rc;
}

int or_amg_aggregates(or_ctx* c, int level, int* agg) {
    if (!c->amg_built) amg_setup(c);
    if (level < 0 || level >= c->nlev - 1) return -1;
    memcpy(agg, c->lev[level].agg, c->lev[level].nnode * sizeof(int));
    return c->lev[level].nagg;
}

/* SolveFem::ComputeObjectiveAndSensitivities (SolveFem.cpp:159-265) */
/* the sums of ComputeObjectiveAndSensitivities (SolveFem.cpp:208-249) for a
 * given displacement U: fx = sum E_e u_e'Ke u_e, dfdx, gx[0], dgdx[0] */
void or_obj_sens_given_u(or_ctx* c, const double* xphys, const double* U, double* fx, double* gx, double* dfdx,
                         double* dgdx) {
    const or_params* p = &c->p;
    int nen = c->nen, nd = c->ndof_e, ne = c->ne;
    double f = 0.0, g = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : f, g)
    for (int e = 0; e < ne; e++) {
        double ue[24];
        for (int cc = 0; cc < 3; cc++)
            for (int l = 0; l < nen; l++) ue[cc * nen + l] = U[3 * c->elem[e * nen + l] + cc];
        const double* ke = c->ke + (size_t)e * nd * nd;
        double uKu = 0.0;
        for (int k = 0; k < nd; k++)
            for (int h = 0; h < nd; h++) uKu += ue[k] * ke[k * nd + h] * ue[h];
        double x = xphys[e];
        f += (p->Emin + pow(x, p->penal) * (p->Emax - p->Emin)) * uKu;
        dfdx[e] = -1.0 * p->penal * pow(x, p->penal - 1) * (p->Emax - p->Emin) * uKu;
        g += x * c->vol[e];
        dgdx[e] = c->vol[e] / c->TV;
    }
    *fx = f;
    for (int i = 0; i < p->m; i++) gx[i] = 0.0;
    gx[0] = g / c->TV - p->volfrac;
}

int or_fem_obj_sens(or_ctx* c, const double* xphys, double* fx, double* gx, double* dfdx, double* dgdx, double* Uout) {
    or_assemble(c, xphys);
    double* U = Uout ? Uout : malloc(c->n * sizeof(double));
    int rc = or_solve(c, U, NULL, NULL);
    or_obj_sens_given_u(c, xphys, U, fx, gx, dfdx, dgdx);
    if (!Uout) free(U);
    return rc;
}

/* ------------------------------------------------------------------ */
/* PDE filter (PDEFilter.cpp)                                           */
/* ------------------------------------------------------------------ */
/* KSPCG + PCJACOBI, preconditioned norm, nonzero initial guess RX
 * (PDEFilter.cpp:117-137): rnorm0 = ||D^-1 b||, converged when
 * ||D^-1 r|| <= max(rtol rnorm0, atol). */
static int filter_cg(or_ctx* c, const double* bvec, double* x) {
    const or_params* p = &c->p;
    int n = c->nn;
    double *r = c->fr, *z = c->fz, *pp = c->fp, *w = c->fw;
    for (int i = 0; i < n; i++) z[i] = bvec[i] / c->fdiag[i];
    double snorm = sqrt(dot(n, z, z));
    double ttol = p->filter_rtol * snorm > p->filter_atol ? p->filter_rtol * snorm : p->filter_atol;
    spmv(&c->KF, x, w);
    for (int i = 0; i < n; i++) r[i] = bvec[i] - w[i];
    for (int i = 0; i < n; i++) z[i] = r[i] / c->fdiag[i];
    double dp = sqrt(dot(n, z, z));
    c->filter_its = 0;
    if (dp <= ttol) return 0;
    double beta = dot(n, z, r), betaold = 0.0, dpi;
    int i = 0;
    do {
        c->filter_its = i + 1;
        if (beta == 0.0) return 0;
        if (i == 0) memcpy(pp, z, n * sizeof(double));
        else { double bb = beta / betaold; for (int q = 0; q < n; q++) pp[q] = z[q] + bb * pp[q]; }
        spmv(&c->KF, pp, w);
        dpi = dot(n, pp, w);
        double a = beta / dpi;
        for (int q = 0; q < n; q++) { x[q] += a * pp[q]; r[q] -= a * w[q]; }
        for (int q = 0; q < n; q++) z[q] = r[q] / c->fdiag[q];
        dp = sqrt(dot(n, z, z));
        if (dp <= ttol) return 0;
        if (dp >= p->filter_dtol * snorm) return 2;
        betaold = beta;
        beta = dot(n, z, r);
        i++;
    } while (i < p->filter_maxit);
    return 1;
}

static void tf_mult(or_ctx* c, const double* x, double* tx) {
    int nen = c->nen;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < c->nn; i++) {
        double t = 0.0;
        for (int q = c->n2e_ptr[i]; q < c->n2e_ptr[i + 1]; q++) {
            int e = c->n2e[q] / nen, l = c->n2e[q] % nen;
            t += c->tf[(size_t)e * nen + l] * x[e];
        }
        tx[i] = t;
    }
}
static void tfx_tmult(or_ctx* c, const double* rx, double* xf) {
    int nen = c->nen;
    double w = 1.0 / (double)nen;
#pragma omp parallel for schedule(static)
    for (int e = 0; e < c->ne; e++) {
        double t = 0.0;
        for (int l = 0; l < nen; l++) t += w * rx[c->elem[e * nen + l]];
        xf[e] = t;
    }
}

/* PDEFilter::Filter (PDEFilter.cpp:142-165) */
int or_filter(or_ctx* c, const double* x, double* xf, double Xmin) {
    tf_mult(c, x, c->TX);
    int rc = filter_cg(c, c->TX, c->RX);
    tfx_tmult(c, c->RX, xf);
    for (int e = 0; e < c->ne; e++) { if (xf[e] < Xmin) xf[e] = Xmin; else if (xf[e] > 1.0) xf[e] = 1.0; }
    return rc;
}

/* PDEFilter::ComputeFilteredSens (PDEFilter.cpp:167-183): same forward
 * chain applied to dfdx and each dgdx, warm-started from the last RX. */
int or_filter_sens(or_ctx* c, double* dfdx, double* dgdx, int m) {
    int rc = 0;
    tf_mult(c, dfdx, c->TX);
    rc |= filter_cg(c, c->TX, c->RX);
    tfx_tmult(c, c->RX, dfdx);
    for (int j = 0; j < m; j++) {
        tf_mult(c, dgdx + (size_t)j * c->ne, c->TX);
        rc |= filter_cg(c, c->TX, c->RX);
        tfx_tmult(c, c->RX, dgdx + (size_t)j * c->ne);
    }
    return rc;
}

void or_filter_state(or_ctx* c, double* RX, int set) {
    if (set) memcpy(c->RX, RX, c->nn * sizeof(double));
    else memcpy(RX, c->RX, c->nn * sizeof(double));
}
int or_filter_last_its(or_ctx* c) { return c->filter_its; }

/* PDEFilter::HeavisideFilter (PDEFilter.cpp:242-293) */
void or_heaviside(or_ctx* c, const double* xf, double* xp, double x0, double beta0, double betamax, int itr,
                  double Xmin, int proj) {
    if (!proj) { memcpy(xp, xf, c->ne * sizeof(double)); return; }
    if (itr < 30) c->beta_proj = beta0;
    else if (itr % 10 == 0) c->beta_proj = betamax < c->beta_tmp + 1 ? betamax : c->beta_tmp + 1;
    double beta = c->beta_proj;
    for (int i = 0; i < c->ne; i++) {
        xp[i] = (tanh(beta * x0) + tanh(beta * (xf[i] - x0))) / (tanh(beta * x0) + tanh(beta * (1 - x0)));
        if (xp[i] < Xmin) xp[i] = Xmin;
    }
    c->beta_tmp = beta;
}

/* PDEFilter::ComputeProjectedSens (PDEFilter.cpp:295-341) */
void or_projected_sens(or_ctx* c, const double* xf, double* dfdx, double* dgdx, int m, double x0) {
    double beta = c->beta_proj;
    for (int i = 0; i < c->ne; i++) {
        double t = tanh(beta * (xf[i] - x0));
        double dx = beta * (1.0 - t * t) / (tanh(beta * x0) + tanh(beta * (1 - x0)));
        dfdx[i] *= dx;
        for (int j = 0; j < m; j++) dgdx[(size_t)j * c->ne + i] *= dx;
    }
}

/* ------------------------------------------------------------------ */
/* MMA (MMA.cpp, Aage's TopOpt_in_PETSc MMA)                            */
/* ------------------------------------------------------------------ */
static double dmax(double a, double b) { return a > b ? a : b; }
static double dmin(double a, double b) { return a < b ? a : b; }

void or_mma_set_outer_movelimit(or_ctx* c, double Xmin, double Xmax, double movlim, const double* x,
                                double* xmin, double* xmax) {
    /* MMA.cpp:370-389 */
    for (int i = 0; i < c->ne; i++) { xmax[i] = dmin(Xmax, x[i] + movlim); xmin[i] = dmax(Xmin, x[i] - movlim); }
}

double or_mma_design_change(or_ctx* c, const double* x, double* xold) {
    /* MMA.cpp:391-410 */
    double ch = 0.0;
    for (int i = 0; i < c->ne; i++) { ch = dmax(ch, fabs(x[i] - xold[i])); xold[i] = x[i]; }
    return ch;
}

static void mma_gensub(or_ctx* c, const double* xv, const double* dfdx, const double* gx, const double* dgdx,
                       const double* xmin, const double* xmax) {
    /* MMA.cpp:506-637 */
    int n = c->ne, m = c->p.m;
    c->mk++;
    if (c->mk < 3) {
        for (int i = 0; i < n; i++) {
            double Lv = 1.0 * xv[i] + (-c->asyminit) * xmax[i];
            Lv += c->asyminit * xmin[i];
            double Uv = 1.0 * xv[i] + c->asyminit * xmax[i];
            Uv += -c->asyminit * xmin[i];
            c->L[i] = Lv; c->U[i] = Uv;
        }
    }
    if (c->mk > 2) {
        for (int i = 0; i < n; i++) {
            double helpvar = (xv[i] - c->xo1[i]) * (c->xo1[i] - c->xo2[i]);
            double gamma = helpvar < 0.0 ? c->asymdec : (helpvar > 0.0 ? c->asyminc : 1.0);
            c->L[i] = xv[i] - gamma * (c->xo1[i] - c->L[i]);
            c->U[i] = xv[i] + gamma * (c->U[i] - c->xo1[i]);
            double xmi = dmax(1.0e-5, xmax[i] - xmin[i]);
            if (c->RobustAsymptotesType == 0) {
                c->L[i] = dmax(c->L[i], xv[i] - 10.0 * xmi);
                c->L[i] = dmin(c->L[i], xv[i] - 0.01 * xmi);
                c->U[i] = dmax(c->U[i], xv[i] + 0.01 * xmi);
                c->U[i] = dmin(c->U[i], xv[i] + 10.0 * xmi);
            } else {
                c->L[i] = dmax(c->L[i], xv[i] - 100.0 * xmi);
                c->L[i] = dmin(c->L[i], xv[i] - 1.0e-4 * xmi);
                c->U[i] = dmax(c->U[i], xv[i] + 1.0e-4 * xmi);
                c->U[i] = dmin(c->U[i], xv[i] + 100.0 * xmi);
                double xmi2 = xmin[i] - 1.0e-5, xma = xmax[i] + 1.0e-5;
                if (xv[i] < xmi2) { c->L[i] = xv[i] - (xma - xv[i]) / 0.9; c->U[i] = xv[i] + (xma - xv[i]) / 0.9; }
                if (xv[i] > xma) { c->L[i] = xv[i] - (xv[i] - xmi2) / 0.9; c->U[i] = xv[i] + (xv[i] - xmi2) / 0.9; }
            }
        }
    }
    double feps = 1.0e-6;
    for (int i = 0; i < n; i++) {
        double Uv = c->U[i], Lv = c->L[i];
        c->alpha[i] = dmax(xmin[i], 0.9 * Lv + 0.1 * xv[i]);
        c->beta[i] = dmin(xmax[i], 0.9 * Uv + 0.1 * xv[i]);
        double dfdxp = dmax(0.0, dfdx[i]), dfdxm = dmax(0.0, -1.0 * dfdx[i]);
        c->p0[i] = pow(Uv - xv[i], 2.0) * (dfdxp + 0.001 * fabs(dfdx[i]) + 0.5 * feps / (Uv - Lv));
        c->q0[i] = pow(xv[i] - Lv, 2.0) * (dfdxm + 0.001 * fabs(dfdx[i]) + 0.5 * feps / (Uv - Lv));
        for (int j = 0; j < m; j++) {
            double g = dgdx[(size_t)j * n + i];
            double gp = dmax(0.0, g), gm = dmax(0.0, -1.0 * g);
            if (c->constraintModification) {
                c->pij[(size_t)j * n + i] = pow(Uv - xv[i], 2.0) * (gp + 0.001 * fabs(g) + 0.5 * feps / (Uv - Lv));
                c->qij[(size_t)j * n + i] = pow(xv[i] - Lv, 2.0) * (gm + 0.001 * fabs(g) + 0.5 * feps / (Uv - Lv));
            } else {
                c->pij[(size_t)j * n + i] = pow(Uv - xv[i], 2.0) * gp;
                c->qij[(size_t)j * n + i] = pow(xv[i] - Lv, 2.0) * gm;
            }
        }
    }
    for (int j = 0; j < m; j++) {
        double bj = 0.0;
        for (int i = 0; i < n; i++) bj += c->pij[(size_t)j * n + i] / (c->U[i] - xv[i]) + c->qij[(size_t)j * n + i] / (xv[i] - c->L[i]);
        c->b[j] = bj;
    }
    for (int j = 0; j < m; j++) c->b[j] += -gx[j];
}

static void mma_xyz(or_ctx* c, double* x) {
    /* MMA.cpp:678-728 */
    int n = c->ne, m = c->p.m;
    double lamai = 0.0;
    for (int i = 0; i < m; i++) {
        if (c->lam[i] < 0.0) c->lam[i] = 0;
        c->y[i] = dmax(0.0, c->lam[i] - c->c[i]);
        lamai += c->lam[i] * c->a[i];
    }
    c->z = dmax(0.0, 10.0 * (lamai - 1.0));
    for (int i = 0; i < n; i++) {
        double pj = c->p0[i], qj = c->q0[i];
        for (int j = 0; j < m; j++) { pj += c->pij[(size_t)j * n + i] * c->lam[j]; qj += c->qij[(size_t)j * n + i] * c->lam[j]; }
        x[i] = (sqrt(pj) * c->L[i] + sqrt(qj) * c->U[i]) / (sqrt(pj) + sqrt(qj));
        if (x[i] < c->alpha[i]) x[i] = c->alpha[i];
        if (x[i] > c->beta[i]) x[i] = c->beta[i];
    }
}

static void mma_dualgrad(or_ctx* c, const double* x) {
    /* MMA.cpp:730-765 */
    int n = c->ne, m = c->p.m;
    for (int j = 0; j < m; j++) {
        double g = 0.0;
        for (int i = 0; i < n; i++) g += c->pij[(size_t)j * n + i] / (c->U[i] - x[i]) + c->qij[(size_t)j * n + i] / (x[i] - c->L[i]);
        c->grad[j] = g;
    }
    for (int j = 0; j < m; j++) c->grad[j] += -c->b[j] - c->a[j] * c->z - c->y[j];
}

static void mma_dualhess(or_ctx* c, const double* x) {
    /* MMA.cpp:767-868 */
    int n = c->ne, m = c->p.m;
    double* H = c->Hess;
    for (int q = 0; q < m * m; q++) H[q] = 0.0;
    double PQ[16];
    for (int i = 0; i < n; i++) {
        double pj = c->p0[i], qj = c->q0[i];
        double Uu = c->U[i] - x[i], Ll = x[i] - c->L[i];
        for (int j = 0; j < m; j++) {
            pj += c->pij[(size_t)j * n + i] * c->lam[j];
            qj += c->qij[(size_t)j * n + i] * c->lam[j];
            PQ[j] = c->pij[(size_t)j * n + i] / pow(Uu, 2.0) - c->qij[(size_t)j * n + i] / pow(Ll, 2.0);
        }
        double df2 = -1.0 / (2.0 * pj / pow(Uu, 3.0) + 2.0 * qj / pow(Ll, 3.0));
        double xp = (sqrt(pj) * c->L[i] + sqrt(qj) * c->U[i]) / (sqrt(pj) + sqrt(qj));
        if (xp < c->alpha[i]) df2 = 0.0;
        if (xp > c->beta[i]) df2 = 0.0;
        for (int a = 0; a < m; a++)
            for (int b = 0; b < m; b++) H[a * m + b] += (PQ[a] * df2) * PQ[b];
    }
    double lamai = 0.0;
    for (int j = 0; j < m; j++) {
        if (c->lam[j] < 0.0) c->lam[j] = 0.0;
        lamai += c->lam[j] * c->a[j];
        if (c->lam[j] > c->c[j]) H[j * m + j] += -1.0;
        H[j * m + j] += -c->mu[j] / c->lam[j];
    }
    if (lamai > 0.0)
        for (int j = 0; j < m; j++) for (int k = 0; k < m; k++) H[j * m + k] += -10.0 * c->a[j] * c->a[k];
    double tr = 0.0;
    for (int i = 0; i < m; i++) tr += H[i * m + i];
    double corr = 1e-4 * tr / m;
    if (-1.0 * corr < 1.0e-7) corr = -1.0e-7;
    for (int i = 0; i < m; i++) H[i * m + i] += corr;
}

static void mma_factor_solve(double* K, double* x, int nn) {
    /* MMA.cpp:936-969: LU without pivoting */
    for (int ss = 0; ss < nn - 1; ss++)
        for (int i = ss + 1; i < nn; i++) {
            K[i * nn + ss] = K[i * nn + ss] / K[ss * nn + ss];
            for (int j = ss + 1; j < nn; j++) K[i * nn + j] = K[i * nn + j] - K[i * nn + ss] * K[ss * nn + j];
        }
    for (int i = 1; i < nn; i++) { double a = 0.0; for (int j = 0; j < i; j++) a = a - K[i * nn + j] * x[j]; x[i] = x[i] + a; }
    x[nn - 1] = x[nn - 1] / K[(nn - 1) * nn + (nn - 1)];
    for (int i = nn - 2; i >= 0; i--) { double a = x[i]; for (int j = i + 1; j < nn; j++) a = a - K[i * nn + j] * x[j]; x[i] = a / K[i * nn + i]; }
}

static double mma_dualres(or_ctx* c, const double* x, double epsi) {
    /* MMA.cpp:890-934 */
    int n = c->ne, m = c->p.m;
    double res[32];
    for (int j = 0; j < m; j++) {
        double r = 0.0;
        for (int i = 0; i < n; i++) r += c->pij[(size_t)j * n + i] / (c->U[i] - x[i]) + c->qij[(size_t)j * n + i] / (x[i] - c->L[i]);
        res[j] = r; res[j + m] = 0.0;
    }
    for (int j = 0; j < m; j++) {
        res[j] += -c->b[j] - c->a[j] * c->z - c->y[j] + c->mu[j];
        res[j + m] += c->mu[j] * c->lam[j] - epsi;
    }
    double nrI = 0.0;
    for (int i = 0; i < 2 * m; i++) if (nrI < fabs(res[i])) nrI = fabs(res[i]);
    return nrI;
}

static void mma_solvedip(or_ctx* c, double* x) {
    /* MMA.cpp:639-676 */
    int m = c->p.m, n = c->ne;
    for (int j = 0; j < m; j++) { c->lam[j] = c->c[j] / 2.0; c->mu[j] = 1.0; }
    double tol = 1.0e-9 * sqrt((double)(m + n));
    double epsi = 1.0, err = 1.0;
    while (epsi > tol) {
        int loop = 0;
        while (err > 0.9 * epsi && loop < 100) {
            loop++;
            mma_xyz(c, x);
            mma_dualgrad(c, x);
            for (int j = 0; j < m; j++) c->grad[j] = -1.0 * c->grad[j] - epsi / c->lam[j];
            mma_dualhess(c, x);
            mma_factor_solve(c->Hess, c->grad, m);
            for (int j = 0; j < m; j++) c->s[j] = c->grad[j];
            for (int i = 0; i < m; i++) c->s[m + i] = -c->mu[i] + epsi / c->lam[i] - c->s[i] * c->mu[i] / c->lam[i];
            /* DualLineSearch (MMA.cpp:870-888) */
            double theta = 1.005;
            for (int i = 0; i < m; i++) {
                if (theta < -1.01 * c->s[i] / c->lam[i]) theta = -1.01 * c->s[i] / c->lam[i];
                if (theta < -1.01 * c->s[i + m] / c->mu[i]) theta = -1.01 * c->s[i + m] / c->mu[i];
            }
            theta = 1.0 / theta;
            for (int i = 0; i < m; i++) { c->lam[i] = c->lam[i] + theta * c->s[i]; c->mu[i] = c->mu[i] + theta * c->s[i + m]; }
            mma_xyz(c, x);
            err = mma_dualres(c, x, epsi);
        }
        epsi = epsi * 0.1;
    }
}

/* MMA::Update (MMA.cpp:483-502) */
int or_mma_update(or_ctx* c, double* xval, const double* dfdx, const double* gx, const double* dgdx,
                  const double* xmin, const double* xmax) {
    mma_gensub(c, xval, dfdx, gx, dgdx, xmin, xmax);
    memcpy(c->xo2, c->xo1, c->ne * sizeof(double));
    memcpy(c->xo1, xval, c->ne * sizeof(double));
    mma_solvedip(c, xval);
    return 0;
}

void or_mma_state(or_ctx* c, double* xo1, double* xo2, double* L, double* U, int* k) {
    size_t b = c->ne * sizeof(double);
    if (xo1) memcpy(xo1, c->xo1, b);
    if (xo2) memcpy(xo2, c->xo2, b);
    if (L) memcpy(L, c->L, b);
    if (U) memcpy(U, c->U, b);
    if (k) *k = c->mk;
}

/* MMA::SetAsymptotes (MMA.cpp:345-353), SetRobustAsymptotesType (MMA.cpp:355-368; any
 * value other than 0 or 1 falls back to 0) and the constraintModification flag
 * (MMA.h:32-35) */
void or_mma_options(or_ctx* c, double asyminit, double asymdec, double asyminc, int robust, int constraint_mod) {
    c->asyminit = asyminit; c->asymdec = asymdec; c->asyminc = asyminc;
    c->RobustAsymptotesType = (robust == 0 || robust == 1) ? robust : 0;
    c->constraintModification = constraint_mod ? 1 : 0;
}

/* the restart constructor MMA(n, m, k, xo1, xo2, U, L) (MMA.cpp:91-176): the
 * history vectors and the iteration counter k are loaded */
void or_mma_restart_set(or_ctx* c, const double* xo1, const double* xo2, const double* U, const double* L, int k) {
    size_t b = c->ne * sizeof(double);
    memcpy(c->xo1, xo1, b); memcpy(c->xo2, xo2, b); memcpy(c->U, U, b); memcpy(c->L, L, b);
    c->mk = k;
}

/* MMA::KKTresidual (MMA.cpp:412-480) with the multipliers of the last
 * Update: per element the stationarity residual of the box-constrained
 * Lagrangian and the two complementarity terms; then the constraint term
 * lam_j (a_j z + y_j - g_j); norm2 is the root of the sum of squares */
void or_mma_kkt_residual(or_ctx* c, const double* x, const double* dfdx, const double* gx, const double* dgdx,
                         const double* xmin, const double* xmax, double* norm2, double* norm_inf) {
    int n = c->ne, m = c->p.m;
    double n2 = 0.0, ni = 0.0;
    for (int i = 0; i < n; i++) {
        double ri = dfdx[i];
        for (int j = 0; j < m; j++) ri += c->lam[j] * dgdx[(size_t)j * n + i];
        double mu_min = 0.0, mu_max = 0.0;
        if (x[i] < xmin[i] + 1.0e-5 && ri > 0.0) mu_min = ri;
        if (x[i] > xmax[i] - 1.0e-5 && ri < 0.0) mu_max = -ri;
        ri += -mu_min + mu_max;
        n2 += ri * ri;
        ni = dmax(fabs(ri), ni);
        double resi = mu_min * (x[i] - xmin[i]);
        n2 += resi * resi;
        ni = dmax(fabs(resi), ni);
        resi = mu_max * (xmax[i] - x[i]);
        n2 += resi * resi;
        ni = dmax(fabs(resi), ni);
    }
    double ri = 0.0;
    for (int j = 0; j < m; j++) ri += c->lam[j] * (c->a[j] * c->z + c->y[j] - gx[j]);
    n2 += ri * ri;
    ni = dmax(fabs(ri), ni);
    *norm2 = sqrt(n2);
    *norm_inf = ni;
}

/* main.cpp:64-119 loop */
int or_run(or_ctx* c, int maxItr, double ch_tol, double* hist, double* xphys_out) {
    const or_params* p = &c->p;
    int ne = c->ne, m = p->m;
    double* X = malloc(ne * sizeof(double));
    double* Xold = malloc(ne * sizeof(double));
    double* XF = malloc(ne * sizeof(double));
    double* XP = malloc(ne * sizeof(double));
    double* df = malloc(ne * sizeof(double));
    double* dg = malloc((size_t)ne * m * sizeof(double));
    double* xmn = malloc(ne * sizeof(double));
    double* xmx = malloc(ne * sizeof(double));
    double* gx = calloc(m, sizeof(double));
    for (int i = 0; i < ne; i++) X[i] = XF[i] = XP[i] = Xold[i] = p->volfrac;
    int itr = 0;
    or_filter(c, X, XF, p->Xmin);
    or_heaviside(c, XF, XP, p->x0, p->beta0, p->betamax, itr, p->Xmin, p->proj);
    double ch = 1.0, fx = 0.0;
    while (itr < maxItr && ch > ch_tol) {
        itr++;
        or_fem_obj_sens(c, XP, &fx, gx, df, dg, NULL);
        if (p->proj) or_projected_sens(c, XF, df, dg, m, p->x0);
        or_filter_sens(c, df, dg, m);
        or_mma_set_outer_movelimit(c, p->Xmin, p->Xmax, p->movlim, X, xmn, xmx);
        or_mma_update(c, X, df, gx, dg, xmn, xmx);
        ch = or_mma_design_change(c, X, Xold);
        or_filter(c, X, XF, p->Xmin);
        or_heaviside(c, XF, XP, p->x0, p->beta0, p->betamax, itr, p->Xmin, p->proj);
        if (hist) { hist[3 * (itr - 1)] = fx; hist[3 * (itr - 1) + 1] = gx[0]; hist[3 * (itr - 1) + 2] = ch; }
    }
    if (xphys_out) memcpy(xphys_out, XP, ne * sizeof(double));
    free(X); free(Xold); free(XF); free(XP); free(df); free(dg); free(xmn); free(xmx); free(gx);
    return itr;
}
