// Runs the two-phase droplet loop of the reference's MAC driver
// (tests/LargeTests/test_mac2d_large.cpp:303-340: level-set advection,
// MinRK2 reinitialisation, curvature, Heaviside, intermediate velocity,
// divergence, GFM pressure solve, projection, dt update) through the drop-in
// classes LevelSetSolver2D / MACSolver2D, written exactly as a user of the
// reference writes it.
//
// usage: droplet_driver <case.bin> <out.bin>
//   case.bin: int32 nx, ny, steps, solver (0 CG, 1 BiCGStab);
//             float64 dx, dy, rho_h, rho_l, mu_h, mu_l, sigma, g, cfl, dt0;
//             float64 ls[(nx+6)*(ny+6)] (padded, x-major like the fields)
//   out.bin:  per step: float64 ls, u, v, ps (padded), then dt_next
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <vector>

#include "levelset2d.h"
#include "mac2d.h"

int main(int argc, char **argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s case.bin out.bin\n", argv[0]);
        return 2;
    }
    FILE *fi = std::fopen(argv[1], "rb");
    if (!fi) return 2;
    int hdr[4];
    double prm[10];
    if (std::fread(hdr, sizeof(int), 4, fi) != 4 || std::fread(prm, sizeof(double), 10, fi) != 10) return 2;
    const int nx = hdr[0], ny = hdr[1], steps = hdr[2], solver = hdr[3], nbc = 3;
    const double dx = prm[0], dy = prm[1], rhoH = prm[2], rhoL = prm[3], muH = prm[4], muL = prm[5];
    const double sigma = prm[6], gConstant = prm[7], cfl = prm[8], dt0 = prm[9];
    const size_t n = (size_t)(nx + 2 * nbc) * (ny + 2 * nbc);
    std::vector<double> ls(n), lsB(n), H(n), HSmooth(n);
    if (std::fread(ls.data(), sizeof(double), n, fi) != n) return 2;
    std::fclose(fi);

    const double L = 1.0, U = 1.0, baseX = 0.0, baseY = 0.0, lenX = nx * dx, lenY = ny * dy;
    auto MSolver = std::make_unique<MACSolver2D>(rhoH, rhoL, muH, muL, gConstant, GAXISENUM2D::Y, L, U, sigma, nx,
                                                 ny, baseX, baseY, lenX, lenY, TIMEORDERENUM::RK3, cfl, 1.0e30,
                                                 steps, 1, nbc, false);
    MSolver->SetBC_U_2D("dirichlet", "dirichlet", "dirichlet", "dirichlet");
    MSolver->SetBC_V_2D("dirichlet", "dirichlet", "dirichlet", "dirichlet");
    MSolver->SetBC_P_2D("neumann", "neumann", "neumann", "neumann");
    MSolver->SetBCConstantUW(0.0);
    MSolver->SetBCConstantUE(0.0);
    MSolver->SetBCConstantUS(0.0);
    MSolver->SetBCConstantUN(0.0);
    MSolver->SetBCConstantVW(0.0);
    MSolver->SetBCConstantVE(0.0);
    MSolver->SetBCConstantVS(0.0);
    MSolver->SetBCConstantVN(0.0);
    MSolver->SetPoissonSolver(solver == 0 ? POISSONTYPE::CG : POISSONTYPE::BICGSTAB);
    MSolver->SetPLTType(PLTTYPE::NONE);
    auto LSolver = std::make_shared<LevelSetSolver2D>(nx, ny, nbc, baseX, baseY, dx, dy);
    MSolver->AllocateVariables();
    MSolver->ApplyBC_U_2D(MSolver->m_u);
    MSolver->ApplyBC_V_2D(MSolver->m_v);
    MSolver->ApplyBC_P_2D(MSolver->m_ps);
    MSolver->ApplyBC_P_2D(MSolver->m_p);
    LSolver->SetBC_P_2D("neumann", "neumann", "neumann", "neumann");
    LSolver->SetBCConstantPW(0.0);
    LSolver->SetBCConstantPE(0.0);
    LSolver->SetBCConstantPS(0.0);
    LSolver->SetBCConstantPN(0.0);
    LSolver->ApplyBC_P_2D(ls);
    MSolver->m_dt = dt0;

    std::vector<double> uhat(n), vhat(n), div(n);
    FILE *fo = std::fopen(argv[2], "wb");
    if (!fo) return 2;
    const int poissonMaxIter = 200000;
    int stat = 0;
    while (MSolver->m_iter < MSolver->kMaxIter) {
        MSolver->m_iter++;
        lsB = ls;
        LSolver->Solve_LevelSet_2D(ls, MSolver->m_u, MSolver->m_v, MSolver->m_dt);
        LSolver->ApplyBC_P_2D(ls);
        LSolver->Reinit_MinRK2_2D(ls);
        LSolver->ApplyBC_P_2D(ls);

        MSolver->UpdateKappa(ls);
        H = MSolver->UpdateHeavisideFunc(ls);
        HSmooth = MSolver->UpdateSmoothHeavisideFunc(ls);
        MSolver->GetIntermediateVel(LSolver, ls, MSolver->m_u, MSolver->m_v, uhat, vhat, HSmooth);
        MSolver->ApplyBC_U_2D(uhat);
        MSolver->ApplyBC_V_2D(vhat);

        div = MSolver->GetDivergence(uhat, vhat);
        MSolver->ApplyBC_P_2D(MSolver->m_ps);
        LSolver->ApplyBC_P_2D(ls);
        stat = MSolver->SolvePoisson(MSolver->m_ps, div, ls, lsB, MSolver->m_u, MSolver->m_v, H, poissonMaxIter);
        if (stat != 0) return 3;
        MSolver->ApplyBC_P_2D(MSolver->m_ps);
        stat = MSolver->UpdateVel(MSolver->m_u, MSolver->m_v, uhat, vhat, MSolver->m_ps, ls, lsB, H);
        if (stat != 0) return 3;
        MSolver->ApplyBC_U_2D(MSolver->m_u);
        MSolver->ApplyBC_V_2D(MSolver->m_v);
        MSolver->m_dt = MSolver->UpdateDt(MSolver->m_u, MSolver->m_v);
        MSolver->m_curTime += MSolver->m_dt;

        std::fwrite(ls.data(), sizeof(double), n, fo);
        std::fwrite(MSolver->m_u.data(), sizeof(double), n, fo);
        std::fwrite(MSolver->m_v.data(), sizeof(double), n, fo);
        std::fwrite(MSolver->m_ps.data(), sizeof(double), n, fo);
        std::fwrite(&MSolver->m_dt, sizeof(double), 1, fo);
    }
    std::fclose(fo);
    return 0;
}
