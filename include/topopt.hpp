// topopt.hpp -- C++ host classes over the C ABI (topo.h), shaped like the
// reference program's classes so that its main.cpp loop ports line by line:
//   OptPara    (OptPara.h:21-62)      options + design vectors on the device
//   SolveFem   (SolveFem.h:12-55)     ComputeObjectiveAndSensitivities, U
//   PDEFilter  (PDEFilter.h:12-56)    Filter, ComputeFilteredSens, Heaviside
//   MMA        (MMA.h:8-119)          SetOuterMovelimit, Update, DesignChange
//   Write2Vtu  (Write2Vtu.h:9-18)     WriteResults
// Vec is a device vector (no PETSc).  Errors: methods return the C-ABI status
// (0 ok, > 0 warning, < 0 error) like PetscErrorCode; CHKERR below mirrors
// CHKERRQ.  Header only; link with libtopo.so.
#pragma once
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "topo.h"

namespace topopt {

#define TOPO_CHKERR(rc)                                                                  \
    do {                                                                                 \
        int rc_ = (rc);                                                                  \
        if (rc_ < 0) {                                                                   \
            std::fprintf(stderr, "topo error %d at %s:%d: %s\n", rc_, __FILE__, __LINE__, \
                         topo_last_error());                                             \
            return rc_;                                                                  \
        }                                                                                \
    } while (0)

// device vector of doubles (PETSc Vec stand-in)
class Vec {
  public:
    Vec() = default;
    explicit Vec(size_t n) { alloc(n); }
    Vec(const Vec&) = delete;
    Vec& operator=(const Vec&) = delete;
    Vec(Vec&& o) noexcept : d_(o.d_), n_(o.n_) { o.d_ = nullptr; o.n_ = 0; }
    ~Vec() { if (d_) topo_device_free(d_); }
    int alloc(size_t n) {
        if (d_) topo_device_free(d_);
        n_ = n;
        return topo_device_alloc(n * sizeof(double), reinterpret_cast<void**>(&d_));
    }
    double* data() const { return d_; }
    size_t size() const { return n_; }
    int set(topo_ctx* c, double v) {
        std::vector<double> h(n_, v);
        return topo_memcpy_h2d(d_, h.data(), n_ * sizeof(double), c);
    }
    int get(topo_ctx* c, std::vector<double>& h) const {
        h.resize(n_);
        return topo_memcpy_d2h(h.data(), d_, n_ * sizeof(double), c);
    }

  private:
    double* d_ = nullptr;
    size_t n_ = 0;
};

// Mesh + BCs (InputMeshData.h:14-41): from the reference's text files or the
// synthetic lattice generator.
struct InputMeshData {
    int nen = 8, n_nodes = 0, n_elems = 0;
    std::vector<double> vertex, load;
    std::vector<int32_t> element, fixedDofs, loadDofs, case_ptr{0, 0};

    int ReadDir(const std::string& dir, int nen_, int n_cases = 1) {
        nen = nen_;
        int nf = 0, nl = 0;
        TOPO_CHKERR(topo_read_mesh_dir(dir.c_str(), nen, n_cases, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                                       &n_nodes, &n_elems, &nf, &nl));
        vertex.resize(3 * (size_t)n_nodes);
        element.resize((size_t)n_elems * nen);
        fixedDofs.resize(nf);
        loadDofs.resize(nl);
        load.resize(nl);
        case_ptr.resize(n_cases + 1);
        return topo_read_mesh_dir(dir.c_str(), nen, n_cases, vertex.data(), element.data(), fixedDofs.data(),
                                  case_ptr.data(), loadDofs.data(), load.data(), &n_nodes, &n_elems, &nf, &nl);
    }
    int Cantilever(int nx, int ny, int nz, int nen_, double jitter, uint64_t seed, int load_mode = 0) {
        nen = nen_;
        int nf = 0, nl = 0;
        TOPO_CHKERR(topo_gen_cantilever(nx, ny, nz, nen, jitter, seed, load_mode, nullptr, nullptr, nullptr, nullptr,
                                        nullptr, &n_nodes, &n_elems, &nf, &nl));
        vertex.resize(3 * (size_t)n_nodes);
        element.resize((size_t)n_elems * nen);
        fixedDofs.resize(nf);
        loadDofs.resize(nl);
        load.resize(nl);
        case_ptr = {0, nl};
        return topo_gen_cantilever(nx, ny, nz, nen, jitter, seed, load_mode, vertex.data(), element.data(),
                                   fixedDofs.data(), loadDofs.data(), load.data(), &n_nodes, &n_elems, &nf, &nl);
    }
};

// OptPara (OptPara.h:21-62): defaults of OptPara.cpp:66-78, `-flag value`
// overrides of OptPara.cpp:92-104 plus -nu (SolveFem.cpp:11).
struct OptPara {
    topo_params p{};
    Vec X, Xold, XFiled, XPhys, dfdx, dgdx, xmin, xmax, Vol;
    double fx = 0.0;
    std::vector<double> gx;
    double &Emin = p.Emin, &Emax = p.Emax, &volfrac = p.volfrac, &penal = p.penal, &rmin = p.rmin;
    double &Xmin = p.Xmin, &Xmax = p.Xmax, &movlim = p.movlim, &x0 = p.x0, &beta0 = p.beta0,
           &betamax = p.betamax;
    int &maxItr = p.maxItr, &m = p.m, &proj = p.proj;

    OptPara() { topo_params_default(&p); }
    void SetUpOpt(int argc, char** argv) {
        for (int i = 1; i + 1 < argc; i++) {
            const char* k = argv[i];
            const char* v = argv[i + 1];
            struct { const char* name; double* d; } dd[] = {{"-Emin", &p.Emin}, {"-Emax", &p.Emax},
                {"-volfrac", &p.volfrac}, {"-penal", &p.penal}, {"-rmin", &p.rmin}, {"-Xmin", &p.Xmin},
                {"-Xmax", &p.Xmax}, {"-movlim", &p.movlim}, {"-x0", &p.x0}, {"-beta0", &p.beta0},
                {"-betamax", &p.betamax}, {"-nu", &p.nu}, {"-fem_rtol", &p.fem_rtol}, {"-ch_tol", &p.ch_tol}};
            for (auto& e : dd)
                if (!std::strcmp(k, e.name)) *e.d = std::atof(v);
            if (!std::strcmp(k, "-maxItr")) p.maxItr = std::atoi(v);
            if (!std::strcmp(k, "-proj")) p.proj = (!std::strcmp(v, "1") || !std::strcmp(v, "true"));
            if (!std::strcmp(k, "-precision")) p.precision = !std::strcmp(v, "mixed") ? TOPO_PREC_MIXED : TOPO_PREC_FP64;
        }
    }
    void PrintSettings() const {
        std::printf("################### Optimization settings ####################\n");
        std::printf("# -rmin: %f\n# -volfrac: %f\n# -penal: %f\n", p.rmin, p.volfrac, p.penal);
        std::printf("# -Emin/-Emax: %e - %e \n# -Xmin/-Xmax: %e - %e \n", p.Emin, p.Emax, p.Xmin, p.Xmax);
        std::printf("# -maxItr: %i\n# -movlim: %f\n# -x0: %f\n# -beta0: %f\n# -betamax: %f\n", p.maxItr, p.movlim,
                    p.x0, p.beta0, p.betamax);
        std::printf("# -proj: %i  (0/1)\n", p.proj);
        std::printf("##############################################################\n");
    }
    // VecCreate + VecSet(volfrac) of OptPara.cpp:120-148
    int SetUp(topo_ctx* c, int n_elems) {
        gx.assign(p.m, 0.0);
        for (Vec* v : {&X, &Xold, &XFiled, &XPhys, &dfdx, &xmin, &xmax, &Vol}) TOPO_CHKERR(v->alloc(n_elems));
        TOPO_CHKERR(dgdx.alloc((size_t)n_elems * p.m));
        for (Vec* v : {&X, &XFiled, &XPhys, &Xold}) TOPO_CHKERR(v->set(c, p.volfrac));
        return 0;
    }
};

class SolveFem {
  public:
    explicit SolveFem(topo_ctx* c) : c_(c) {}
    // SolveFem::SolveFem fills Vol (SolveFem.cpp:6-15)
    int ComputeTotalVol(Vec& Vol, double* TV) { return topo_fem_volumes(c_, Vol.data(), TV); }
    int ComputeObjectiveAndSensitivities(double* fx, double* gx, Vec& dfdx, Vec& dgdx, const Vec& XPhys) {
        return topo_fem_obj_sens(c_, XPhys.data(), fx, gx, dfdx.data(), dgdx.data());
    }
    int U(Vec& out) { return topo_fem_displacement(c_, out.data()); }

  private:
    topo_ctx* c_;
};

class PDEFilter {
  public:
    explicit PDEFilter(topo_ctx* c) : c_(c) {}
    int Filter(const Vec& X, Vec& XFiled, double Xmin) { return topo_filter_apply(c_, X.data(), XFiled.data(), Xmin); }
    int ComputeFilteredSens(Vec& dfdx, Vec& dgdx, int m) { return topo_filter_sens(c_, dfdx.data(), dgdx.data(), m); }
    int HeavisideFilter(const Vec& XFiled, Vec& XPhys, double x0, double beta0, double betamax, int itr, double Xmin,
                        int proj) {
        return topo_heaviside(c_, XFiled.data(), XPhys.data(), x0, beta0, betamax, itr, Xmin, proj);
    }
    int ComputeProjectedSens(const Vec& XFiled, Vec& dfdx, Vec& dgdx, int m, double x0) {
        return topo_projected_sens(c_, XFiled.data(), dfdx.data(), dgdx.data(), m, x0);
    }

  private:
    topo_ctx* c_;
};

class MMA {
  public:
    explicit MMA(topo_ctx* c) : c_(c) {}
    int SetOuterMovelimit(double Xmin, double Xmax, double movlim, const Vec& x, Vec& xmin, Vec& xmax) {
        return topo_mma_set_outer_movelimit(c_, Xmin, Xmax, movlim, x.data(), xmin.data(), xmax.data());
    }
    int Update(Vec& xval, const Vec& dfdx, const double* gx, const Vec& dgdx, const Vec& xmin, const Vec& xmax) {
        return topo_mma_update(c_, xval.data(), dfdx.data(), gx, dgdx.data(), xmin.data(), xmax.data());
    }
    // MMA::DesignChange (MMA.cpp:391-410) returns ch; here ch comes back
    // through the out-parameter and the status is returned, so that a failed
    // call reaches the caller's TOPO_CHKERR instead of looking like a
    // converged design
    int DesignChange(const Vec& x, Vec& xold, double* ch) {
        return topo_mma_design_change(c_, x.data(), xold.data(), ch);
    }
    int SetAsymptotes(double init, double decrease, double increase) {
        return topo_mma_set_asymptotes(c_, init, decrease, increase);
    }

  private:
    topo_ctx* c_;
};

class Write2Vtu {
  public:
    explicit Write2Vtu(topo_ctx* c, std::string dir = ".") : c_(c), dir_(std::move(dir)) {}
    int WriteResults(const Vec& XPhys, int itr) { return topo_write_vtu(c_, dir_.c_str(), itr, XPhys.data()); }

  private:
    topo_ctx* c_;
    std::string dir_;
};

}  // namespace topopt
