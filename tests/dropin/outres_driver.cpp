// Writes Tecplot ASCII output through the drop-in MACSolver2D::OutRes, the
// way the reference's drivers call it (SetPLTType, then OutRes per output
// step with m_iter counting the steps).
//
// usage: outres_driver <case.bin> <vel_base> <div_base>
//   case.bin: int32 nx, ny, zones; float64 base_x, base_y, len_x, len_y;
//             per zone: float64 t, then u, v, ps, ls (padded (nx+6)*(ny+6))
#include <cstdio>
#include <memory>
#include <vector>

#include "mac2d.h"

int main(int argc, char **argv) {
    if (argc != 4) {
        std::fprintf(stderr, "usage: %s case.bin vel_base div_base\n", argv[0]);
        return 2;
    }
    FILE *fi = std::fopen(argv[1], "rb");
    if (!fi) return 2;
    int hdr[3];
    double geo[4];
    if (std::fread(hdr, sizeof(int), 3, fi) != 3 || std::fread(geo, sizeof(double), 4, fi) != 4) return 2;
    const int nx = hdr[0], ny = hdr[1], zones = hdr[2], nbc = 3;
    const size_t n = (size_t)(nx + 2 * nbc) * (ny + 2 * nbc);
    auto MSolver = std::make_unique<MACSolver2D>(1000.0, 1.0, 1e-3, 1e-5, 9.8, GAXISENUM2D::Y, 1.0, 1.0, 0.0728,
                                                 nx, ny, geo[0], geo[1], geo[2], geo[3], TIMEORDERENUM::RK3, 0.5,
                                                 1.0e30, 1 << 30, 1, nbc, false);
    MSolver->SetBC_U_2D("dirichlet", "dirichlet", "dirichlet", "dirichlet");
    MSolver->SetBC_V_2D("dirichlet", "dirichlet", "dirichlet", "dirichlet");
    MSolver->SetBC_P_2D("neumann", "neumann", "neumann", "neumann");
    MSolver->AllocateVariables();
    MSolver->SetPLTType(PLTTYPE::ASCII);
    std::vector<double> u(n), v(n), ps(n), ls(n);
    for (int z = 0; z < zones; z++) {
        double t;
        if (std::fread(&t, sizeof(double), 1, fi) != 1 || std::fread(u.data(), sizeof(double), n, fi) != n ||
            std::fread(v.data(), sizeof(double), n, fi) != n || std::fread(ps.data(), sizeof(double), n, fi) != n ||
            std::fread(ls.data(), sizeof(double), n, fi) != n)
            return 2;
        MSolver->m_iter = z;
        MSolver->OutRes(z, t, argv[2], argv[3], u, v, ps, ls);
    }
    std::fclose(fi);
    return 0;
}
