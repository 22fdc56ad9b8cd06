// Internal to the drop-in classes: a lazily (re)created asd2g session whose
// parameters follow the owning object's configuration, and host<->device
// helpers for the std::vector fields of the reference interfaces.
#ifndef ASD2_DROPIN_SESSION_H
#define ASD2_DROPIN_SESSION_H

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "asd2g.h"
#include "common.h"

class BoundaryCondition2D;

namespace asd2g_dropin {

int bc_code(BC2D b);

// Fill the boundary part of asd2g_params from a BoundaryCondition2D.
void params_from_bc(const BoundaryCondition2D &bc, asd2g_params &p);

struct SessionCache {
    asd2g_session *s = nullptr;
    asd2g_params p{};
    ~SessionCache();
    // Returns the session for these parameters, recreating it when they changed.
    asd2g_session *get(const asd2g_params &want);
    void up(int field, const std::vector<double> &v);
    void down(int field, std::vector<double> &v);
};

// One Tecplot ASCII zone of OutRes (mac2d.cpp:1990-2063, mac2dAxisym.cpp:2323-
// 2397): the cell-centred interior, x fastest, "x,y,c0,c1,..." per cell with
// an ostream's default double format; header (TITLE / VARIABLES) when asked.
bool write_zone(const std::string &path, bool header, const char *title, const char *vars, int iter, double t,
                int nx, int ny, int nbc, double base_x, double base_y, double dx, double dy,
                const std::vector<const std::vector<double> *> &cols);

// Report a failed call the way the reference reports errors: a message; for
// a non-finite value, exit(1) as the reference does on NaN/Inf.
int report(int rc, const char *what);

}  // namespace asd2g_dropin
#endif
