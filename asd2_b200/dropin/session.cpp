#include "session.h"

#include <cstdio>
#include <string>

#include "bc2d.h"

namespace asd2g_dropin {

int bc_code(BC2D b) { return static_cast<int>(b); }

void params_from_bc(const BoundaryCondition2D &bc, asd2g_params &p) {
    const BC2D u[4] = {bc.m_BC_UW, bc.m_BC_UE, bc.m_BC_US, bc.m_BC_UN};
    const BC2D v[4] = {bc.m_BC_VW, bc.m_BC_VE, bc.m_BC_VS, bc.m_BC_VN};
    const BC2D q[4] = {bc.m_BC_PW, bc.m_BC_PE, bc.m_BC_PS, bc.m_BC_PN};
    const double cu[4] = {bc.m_BC_DirichletConstantUW, bc.m_BC_DirichletConstantUE, bc.m_BC_DirichletConstantUS,
                          bc.m_BC_DirichletConstantUN};
    const double cv[4] = {bc.m_BC_DirichletConstantVW, bc.m_BC_DirichletConstantVE, bc.m_BC_DirichletConstantVS,
                          bc.m_BC_DirichletConstantVN};
    const double cp[4] = {bc.m_BC_DirichletConstantPW, bc.m_BC_DirichletConstantPE, bc.m_BC_DirichletConstantPS,
                          bc.m_BC_DirichletConstantPN};
    for (int k = 0; k < 4; k++) {
        p.bc_u[k] = bc_code(u[k]);
        p.bc_v[k] = bc_code(v[k]);
        p.bc_p[k] = bc_code(q[k]);
        p.bcc_u[k] = cu[k];
        p.bcc_v[k] = cv[k];
        p.bcc_p[k] = cp[k];
    }
}

SessionCache::~SessionCache() {
    if (s) asd2g_destroy(s);
}

asd2g_session *SessionCache::get(const asd2g_params &want) {
    if (s && std::memcmp(&want, &p, sizeof(asd2g_params)) == 0) return s;
    if (s) asd2g_destroy(s);
    s = nullptr;
    p = want;
    const int rc = asd2g_create(&p, nullptr, &s);
    if (rc != ASD2G_OK) {
        std::fprintf(stderr, "asd2g: session creation failed: %s\n", asd2g_last_error());
        s = nullptr;
    }
    return s;
}

void SessionCache::up(int field, const std::vector<double> &v) {
    if (!s || v.size() < (size_t)(p.nx + 6) * (p.ny + 6)) {
        std::fprintf(stderr, "asd2g upload: no session or array smaller than (nx+6)*(ny+6)\n");
        return;
    }
    report(asd2g_upload(s, field, v.data()), "upload");
}

void SessionCache::down(int field, std::vector<double> &v) {
    if (!s || v.size() < (size_t)(p.nx + 6) * (p.ny + 6)) {
        std::fprintf(stderr, "asd2g download: no session or array smaller than (nx+6)*(ny+6)\n");
        return;
    }
    report(asd2g_download(s, field, v.data()), "download");
}

int report(int rc, const char *what) {
    if (rc >= 0) return rc;
    std::fprintf(stderr, "asd2g %s failed (%d): %s\n", what, rc, asd2g_last_error());
    if (rc == ASD2G_E_NONFINITE) std::exit(1);
    return rc;
}

// One Tecplot ASCII zone (point packing, x fastest) of the cell-centred
// interior: a zone line, then per cell "x,y,c0,c1,c2" with the values
// formatted as an ostream's default double output (%g, 6 significant digits).
bool write_zone(const std::string &path, bool header, const char *title, const char *vars, int iter, double t,
                int nx, int ny, int nbc, double base_x, double base_y, double dx, double dy,
                const std::vector<const std::vector<double> *> &cols) {
    std::FILE *f = std::fopen(path.c_str(), header ? "w" : "a");
    if (!f) return false;
    if (header) std::fprintf(f, "TITLE = %s\nVARIABLES = %s \n", title, vars);
    std::fprintf(f, "ZONE T=\"%d\", I=%d, J=%d, SOLUTIONTIME=%g, STRANDID=%d\n", iter, nx, ny, t, iter + 1);
    const int64_t stride = ny + 2 * nbc;
    std::string line;
    char num[40];
    for (int j = nbc; j < ny + nbc; j++)
        for (int i = nbc; i < nx + nbc; i++) {
            const int64_t k = j + stride * i;
            line.clear();
            std::snprintf(num, sizeof num, "%g", base_x + static_cast<double>(i + 0.5 - nbc) * dx);
            line += num;
            std::snprintf(num, sizeof num, ",%g", base_y + static_cast<double>(j + 0.5 - nbc) * dy);
            line += num;
            for (const std::vector<double> *c : cols) {
                std::snprintf(num, sizeof num, ",%g", (*c)[k]);
                line += num;
            }
            line += '\n';
            std::fputs(line.c_str(), f);
        }
    return std::fclose(f) == 0;
}

}  // namespace asd2g_dropin
