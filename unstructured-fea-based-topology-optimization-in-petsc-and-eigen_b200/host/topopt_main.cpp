// topopt_main.cpp -- the reference's main.cpp optimisation loop (main.cpp:35-137)
// on the sm_100a library, through the C++ classes of topopt.hpp.
//
//   topopt -mesh_dir DIR [-nen 8|4]            reference text files (InputMeshData.cpp)
//   topopt -lattice NX NY NZ [-nen 8|4]        seeded synthetic cantilever
//   options as the reference: -Emin -Emax -volfrac -penal -rmin -maxItr -Xmin
//   -Xmax -movlim -x0 -beta0 -betamax -proj -nu, plus -precision fp64|mixed,
//   -vtu DIR (write output_initial / output_<20k> / output_final .vtu).
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>

#include "topopt.hpp"

using namespace topopt;

int main(int argc, char** argv) {
    auto t_ini = std::chrono::steady_clock::now();
    OptPara opt;
    opt.SetUpOpt(argc, argv);
    InputMeshData mesh;
    int nen = 8, nx = 0, ny = 0, nz = 0;
    std::string mesh_dir, vtu_dir;
    for (int i = 1; i < argc; i++) {
        if (!std::strcmp(argv[i], "-nen") && i + 1 < argc) nen = std::atoi(argv[i + 1]);
        if (!std::strcmp(argv[i], "-mesh_dir") && i + 1 < argc) mesh_dir = argv[i + 1];
        if (!std::strcmp(argv[i], "-vtu") && i + 1 < argc) vtu_dir = argv[i + 1];
        if (!std::strcmp(argv[i], "-lattice") && i + 3 < argc) {
            nx = std::atoi(argv[i + 1]);
            ny = std::atoi(argv[i + 2]);
            nz = std::atoi(argv[i + 3]);
        }
    }
    opt.PrintSettings();
    int rc = !mesh_dir.empty() ? mesh.ReadDir(mesh_dir, nen)
                               : mesh.Cantilever(nx ? nx : 40, ny ? ny : 20, nz ? nz : 10, nen, nen == 8 ? 0.1 : 0.2,
                                                 2024);
    TOPO_CHKERR(rc);
    topo_ctx* ctx = nullptr;
    TOPO_CHKERR(topo_create(&opt.p, mesh.nen, mesh.n_nodes, mesh.vertex.data(), mesh.n_elems, mesh.element.data(),
                            (int)mesh.fixedDofs.size(), mesh.fixedDofs.data(), 1, mesh.case_ptr.data(),
                            mesh.loadDofs.data(), mesh.load.data(), nullptr, &ctx));
    TOPO_CHKERR(opt.SetUp(ctx, mesh.n_elems));
    SolveFem fem(ctx);
    double TV = 0.0;
    TOPO_CHKERR(fem.ComputeTotalVol(opt.Vol, &TV));
    PDEFilter pde(ctx);
    MMA mma(ctx);
    Write2Vtu vtu(ctx, vtu_dir.empty() ? "." : vtu_dir);
    int itr = 0;
    TOPO_CHKERR(pde.Filter(opt.X, opt.XFiled, opt.Xmin));
    TOPO_CHKERR(pde.HeavisideFilter(opt.XFiled, opt.XPhys, opt.x0, opt.beta0, opt.betamax, itr, opt.Xmin, opt.proj));
    double ch = 1.0;
    const double ch_tol = opt.p.ch_tol;
    while (itr < opt.maxItr && (ch_tol <= 0 || ch > ch_tol)) {
        itr++;
        auto t1 = std::chrono::steady_clock::now();
        TOPO_CHKERR(fem.ComputeObjectiveAndSensitivities(&opt.fx, opt.gx.data(), opt.dfdx, opt.dgdx, opt.XPhys));
        if (itr == 1 && !vtu_dir.empty()) TOPO_CHKERR(vtu.WriteResults(opt.XPhys, 0));
        if (opt.proj) TOPO_CHKERR(pde.ComputeProjectedSens(opt.XFiled, opt.dfdx, opt.dgdx, opt.m, opt.x0));
        TOPO_CHKERR(pde.ComputeFilteredSens(opt.dfdx, opt.dgdx, opt.m));
        TOPO_CHKERR(mma.SetOuterMovelimit(opt.Xmin, opt.Xmax, opt.movlim, opt.X, opt.xmin, opt.xmax));
        TOPO_CHKERR(mma.Update(opt.X, opt.dfdx, opt.gx.data(), opt.dgdx, opt.xmin, opt.xmax));
        TOPO_CHKERR(mma.DesignChange(opt.X, opt.Xold, &ch));
        TOPO_CHKERR(pde.Filter(opt.X, opt.XFiled, opt.Xmin));
        TOPO_CHKERR(pde.HeavisideFilter(opt.XFiled, opt.XPhys, opt.x0, opt.beta0, opt.betamax, itr, opt.Xmin, opt.proj));
        double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
        std::printf("It.: %i, fx: %f, gx[0]: %f, ch.: %f, time: %f\n", itr, opt.fx, opt.gx[0], ch, dt);
        if (itr % 20 == 0 && !vtu_dir.empty()) TOPO_CHKERR(vtu.WriteResults(opt.XPhys, itr));
    }
    if (!vtu_dir.empty()) TOPO_CHKERR(vtu.WriteResults(opt.XPhys, -1));
    topo_destroy(ctx);
    double total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_ini).count();
    std::printf("total time: %f hours\n", total / 3600.0);
    return 0;
}
