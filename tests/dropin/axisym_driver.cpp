// Runs the reference's axisymmetric driver loop
// (tests/LargeTests/test_mac2d_large.cpp:1145-1306: level-set advection and
// MinRK2 reinitialisation with the level set's own boundary object, the
// axisymmetric curvature, Heaviside, GetRHSU / GetUHat / GetRHSV / GetVHat,
// GetDivergence4Poisson, SolvePoisson with the reference CG, UpdateVel,
// UpdateDt) through the drop-in classes LevelSetSolver2D / MACSolver2DAxisym,
// written as a user of the reference writes it.
//
// usage: axisym_driver <case.bin> <out.bin>
//   case.bin: int32 nr, nz, steps, kind (0: the NonSurfaceTension flow,
//             1: a stationary bubble with surface tension);
//             float64 lenR, lenZ, rho_h, rho_l, mu_h, mu_l, sigma, cfl, u0;
//             float64 ls[(nr+6)*(nz+6)] (padded, r-major like the fields)
//   out.bin:  per step: float64 ls, u, v, ps (padded), then dt_next
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <vector>

#include "levelset2d.h"
#include "mac2dAxisym.h"

int main(int argc, char **argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s case.bin out.bin\n", argv[0]);
        return 2;
    }
    FILE *fi = std::fopen(argv[1], "rb");
    if (!fi) return 2;
    int hdr[4];
    double prm[9];
    if (std::fread(hdr, sizeof(int), 4, fi) != 4 || std::fread(prm, sizeof(double), 9, fi) != 9) return 2;
    const int nr = hdr[0], nz = hdr[1], steps = hdr[2], kind = hdr[3], nbc = 3;
    const double lenR = prm[0], lenZ = prm[1], rhoH = prm[2], rhoL = prm[3], muH = prm[4], muL = prm[5];
    const double sigma = prm[6], cfl = prm[7], u0 = prm[8];
    const size_t n = (size_t)(nr + 2 * nbc) * (nz + 2 * nbc);
    std::vector<double> ls(n), lsB(n), H(n), HSmooth(n);
    if (std::fread(ls.data(), sizeof(double), n, fi) != n) return 2;
    std::fclose(fi);

    const double L = 1.0, U = 1.0, baseR = 0.0, baseZ = 0.0, gConstant = 0.0;
    const double dr = lenR / nr, dz = lenZ / nz;
    const int poissonMaxIter = 10000;
    auto MSolver = std::make_unique<MACSolver2DAxisym>(rhoH, rhoL, muH, muL, gConstant, GAXISENUM2DAXISYM::Z, L, U,
                                                       sigma, nr, nz, baseR, baseZ, lenR, lenZ, cfl, 1.0e30, steps, 1,
                                                       nbc, false);
    if (kind == 0) {
        MSolver->SetBC_U_2D("axisym", "neumann", "dirichlet", "dirichlet");
        MSolver->SetBC_V_2D("axisym", "neumann", "dirichlet", "dirichlet");
        MSolver->SetBC_P_2D("axisym", "pressure", "neumann", "neumann");
        MSolver->SetBCConstantUE(1.0);
        MSolver->SetBCConstantUS(1.0);
        MSolver->SetBCConstantUN(1.0);
    } else {
        MSolver->SetBC_U_2D("axisym", "wall", "neumann", "neumann");
        MSolver->SetBC_V_2D("axisym", "wall", "neumann", "neumann");
        MSolver->SetBC_P_2D("axisym", "wall", "neumann", "outlet");
        MSolver->SetBCConstantUE(0.0);
        MSolver->SetBCConstantUS(0.0);
        MSolver->SetBCConstantUN(0.0);
    }
    MSolver->SetBCConstantVE(0.0);
    MSolver->SetBCConstantVS(0.0);
    MSolver->SetBCConstantVN(0.0);
    MSolver->SetPLTType(PLTTYPE::NONE);
    MSolver->SetPoissonSolver(POISSONTYPE::CG);

    auto LSolver = std::make_shared<LevelSetSolver2D>(nr, nz, nbc, baseR, baseZ, dr, dz);
    MSolver->AllocateVariables();
    LSolver->SetBC_P_2D("axisym", "lsfree", "lsfree", "lsfree");
    LSolver->SetBCConstantPW(0.0);
    LSolver->SetBCConstantPE(0.0);
    LSolver->SetBCConstantPS(0.0);
    LSolver->SetBCConstantPN(0.0);
    LSolver->ApplyBC_P_2D(ls);
    LSolver->Reinit_MinRK2_2D(ls);
    LSolver->ApplyBC_P_2D(ls);

    for (size_t k = 0; k < n; k++) {
        MSolver->m_u[k] = u0;
        MSolver->m_v[k] = 0.0;
        MSolver->m_p[k] = 0.0;
        MSolver->m_ps[k] = 0.0;
    }
    MSolver->m_dt = cfl * std::min(dr, dz) / U;
    // UpdateDt of a fluid at rest has no bound; the driver keeps cfl dx / U then
    if (u0 != 0.0) MSolver->m_dt = MSolver->UpdateDt(MSolver->m_u, MSolver->m_v);
    MSolver->UpdateAmbientPressure(0.0);
    MSolver->ApplyBC_U_2D(MSolver->m_u);
    MSolver->ApplyBC_V_2D(MSolver->m_v);
    MSolver->ApplyBC_P_2D(MSolver->m_ps);

    FILE *fo = std::fopen(argv[2], "wb");
    if (!fo) return 2;
    std::vector<double> uhat(n), vhat(n), rhsU(n), rhsV(n), div(n);
    for (int it = 0; it < steps; it++) {
        MSolver->m_iter++;
        lsB = ls;
        LSolver->Solve_LevelSet_2D(ls, MSolver->m_u, MSolver->m_v, MSolver->m_dt);
        LSolver->ApplyBC_P_2D(ls);
        LSolver->Reinit_MinRK2_2D(ls);
        LSolver->ApplyBC_P_2D(ls);

        MSolver->UpdateKappa(ls);
        H = MSolver->UpdateHeavisideFunc(ls);
        HSmooth = MSolver->UpdateSmoothHeavisideFunc(ls);

        rhsU = MSolver->GetRHSU(ls, MSolver->m_u, MSolver->m_v, HSmooth);
        uhat = MSolver->GetUHat(ls, MSolver->m_u, rhsU, HSmooth);
        MSolver->ApplyBC_U_2D(uhat);
        rhsV = MSolver->GetRHSV(ls, MSolver->m_u, uhat, MSolver->m_v, HSmooth);
        vhat = MSolver->GetVHat(ls, MSolver->m_v, rhsV, HSmooth);
        MSolver->ApplyBC_V_2D(vhat);

        div = MSolver->GetDivergence4Poisson(uhat, vhat);
        LSolver->ApplyBC_P_2D(ls);
        MSolver->SolvePoisson(MSolver->m_ps, div, ls, lsB, MSolver->m_u, MSolver->m_v, H, poissonMaxIter);
        MSolver->ApplyBC_P_2D(MSolver->m_ps);
        MSolver->UpdateVel(MSolver->m_u, MSolver->m_v, uhat, vhat, MSolver->m_ps, ls, lsB, H);
        MSolver->ApplyBC_U_2D(MSolver->m_u);
        MSolver->ApplyBC_V_2D(MSolver->m_v);

        MSolver->m_dt = MSolver->UpdateDt(MSolver->m_u, MSolver->m_v);
        MSolver->m_curTime += MSolver->m_dt;
        MSolver->UpdateAmbientPressure(0.0);

        std::fwrite(ls.data(), sizeof(double), n, fo);
        std::fwrite(MSolver->m_u.data(), sizeof(double), n, fo);
        std::fwrite(MSolver->m_v.data(), sizeof(double), n, fo);
        std::fwrite(MSolver->m_ps.data(), sizeof(double), n, fo);
        std::fwrite(&MSolver->m_dt, sizeof(double), 1, fo);
    }
    std::fclose(fo);
    return 0;
}
