// Per-cell arithmetic of the level-set and momentum stencils, in the
// reference's operation order.  Built with -fmad=false so that no product is
// fused into an add: every +, -, *, / and sqrt below rounds exactly as the
// reference's x86-64 build does, which makes the FP64 results bit-identical
// to the reference wherever no cos/sin/pow(x,3) is involved.
#pragma once
#include "internal.cuh"

namespace asd2g {

constexpr double kPi = 3.14159265358979323846;  // the value of M_PI

__device__ __forceinline__ double sq(double x) { return x * x; }
__device__ __forceinline__ int isgn(double v) { return (v > 0) - (v < 0); }
// std::max / std::min semantics
__device__ __forceinline__ double smax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double smin(double a, double b) { return (b < a) ? b : a; }

// LevelSetSolver2D::MinMod, levelset2d.cpp:1036-1046
__device__ __forceinline__ double minmod(double a, double b) {
    const double p = a * b;
    if ((fabs(a) <= fabs(b)) && (p > 0)) return a;
    if ((fabs(a) > fabs(b)) && (p > 0)) return b;
    if (p <= 0) return 0.0;
    return __longlong_as_double(0x7ff8000000000000ULL);
}

// UnitHJWENO5 at one point (levelset2d.cpp:159-262).  D[k] = DFPlus[i-3+k],
// k = 0..5.  dv divides by the spacing d.
__device__ __forceinline__ void weno5_point(const double D[6], const DivH &dv, double &FP, double &FM) {
    const double eps = 1e-6;
    // phi^- uses DFPlus[i-3 .. i+1]
    {
        const double d3 = D[0], d2 = D[1], d1 = D[2], d0 = D[3], p1 = D[4];
        const double is0 = 13.0 / 12.0 * sq(dv(d3 - 2.0 * d2 + d1)) + 1.0 / 4.0 * sq(dv(d3 - 4.0 * d2 + 3.0 * d1));
        const double is1 = 13.0 / 12.0 * sq(dv(d2 - 2.0 * d1 + d0)) + 1.0 / 4.0 * sq(dv(d2 - d0));
        const double is2 = 13.0 / 12.0 * sq(dv(d1 - 2.0 * d0 + p1)) + 1.0 / 4.0 * sq(dv(3.0 * d1 - 4.0 * d0 + p1));
        const double a0 = 0.1 / sq(eps + is0), a1 = 0.6 / sq(eps + is1), a2 = 0.3 / sq(eps + is2);
        const double w0 = a0 / (a0 + a1 + a2), w1 = a1 / (a0 + a1 + a2), w2 = a2 / (a0 + a1 + a2);
        FM = dv(w0 * (1.0 / 3.0 * d3 - 7.0 / 6.0 * d2 + 11.0 / 6.0 * d1)) +
             dv(w1 * (-1.0 / 6.0 * d2 + 5.0 / 6.0 * d1 + 1.0 / 3.0 * d0)) +
             dv(w2 * (1.0 / 3.0 * d1 + 5.0 / 6.0 * d0 - 1.0 / 6.0 * p1));
    }
    // phi^+ uses DFPlus[i-2 .. i+2]
    {
        const double m2 = D[1], m1 = D[2], d0 = D[3], p1 = D[4], p2 = D[5];
        const double is0 = 13.0 / 12.0 * sq(dv(p2 - 2.0 * p1 + d0)) + 1.0 / 4.0 * sq(dv(p2 - 4.0 * p1 + 3.0 * d0));
        const double is1 = 13.0 / 12.0 * sq(dv(p1 - 2.0 * d0 + m1)) + 1.0 / 4.0 * sq(dv(p1 - m1));
        const double is2 = 13.0 / 12.0 * sq(dv(d0 - 2.0 * m1 + m2)) + 1.0 / 4.0 * sq(dv(3.0 * d0 - 4.0 * m1 + m2));
        const double a0 = 0.1 / sq(eps + is0), a1 = 0.6 / sq(eps + is1), a2 = 0.3 / sq(eps + is2);
        const double w0 = a0 / (a0 + a1 + a2), w1 = a1 / (a0 + a1 + a2), w2 = a2 / (a0 + a1 + a2);
        FP = dv(w0 * (1.0 / 3.0 * p2 - 7.0 / 6.0 * p1 + 11.0 / 6.0 * d0)) +
             dv(w1 * (-1.0 / 6.0 * p1 + 5.0 / 6.0 * d0 + 1.0 / 3.0 * m1)) +
             dv(w2 * (1.0 / 3.0 * d0 + 5.0 / 6.0 * m1 - 1.0 / 6.0 * m2));
    }
}

// Signed-velocity blend (HJWENO5_LS_2D :144-154; AddConvectionFU :367-371).
__device__ __forceinline__ double weno_blend(double xp, double xm, double yp, double ym, double ax, double ay) {
    return 0.5 * (xp + xm) + 0.5 * (yp + ym) - ax * (0.5 * (xp - xm)) - ay * (0.5 * (yp - ym));
}

// Second-order ENO one-sided differences along one axis from five values
// c[-2..2] (ENO_DerivAbsLS_2D :567-594).  dh divides by h, dh2 by h*h.
__device__ __forceinline__ void eno_1d(double lm2, double lm1, double l0, double lp1, double lp2, double h,
                                       const DivH &dh, const DivH &dh2, double &dP, double &dM) {
    dP = dh(lp1 - l0) - h * 0.5 * minmod(dh2(lm1 - 2.0 * l0 + lp1), dh2(l0 - 2.0 * lp1 + lp2));
    dM = dh(l0 - lm1) + h * 0.5 * minmod(dh2(lm1 - 2.0 * l0 + lp1), dh2(lm2 - 2.0 * lm1 + l0));
}

// Min-Gibou subcell derivative at a cell whose + neighbour changes sign in
// phi0 (levelset2d.cpp:655-681).  c = phi at the cell; i0m1..i0p2 = phi0.
__device__ __forceinline__ double subcell_plus(double h, const DivH &dh, const DivH &dh2, double c, double i0m1,
                                               double i00, double i0p1, double i0p2) {
    const double DD = minmod(dh2(i0m1 - 2.0 * i00 + i0p1), dh2(i00 - 2.0 * i0p1 + i0p2));
    const double c2 = 0.5 * DD;
    const double c1 = dh(i0p1 - i00);
    const double c0 = (i0p1 + i00) * 0.5 - c2 * h * h * 0.25;
    double nd;
    if (fabs(c2) > 1.0e-10)
        nd = 0.5 * h + (-c1 - isgn(i00) * sqrt(c1 * c1 - 4.0 * c2 * c0)) / (2.0 * c2);
    else
        nd = 0.5 * h - c0 / c1;
    double d = -c / nd - 0.5 * nd * DD;
    if (fabs(nd) < h * 0.01) d = -0.5 * nd * DD;
    return d;
}

// ... and at a cell whose - neighbour changes sign (:686-711).
__device__ __forceinline__ double subcell_minus(double h, const DivH &dh, const DivH &dh2, double c, double i0m2,
                                                double i0m1, double i00, double i0p1) {
    const double DD = minmod(dh2(i0m1 - 2.0 * i00 + i0p1), dh2(i0m2 - 2.0 * i0m1 + i00));
    const double c2 = 0.5 * DD;
    const double c1 = dh(i00 - i0m1);
    const double c0 = (i00 + i0m1) * 0.5 - c2 * h * h * 0.25;
    double nd;
    if (fabs(c2) > 1.0e-10)
        nd = 0.5 * h - (-c1 + isgn(i00) * sqrt(c1 * c1 - 4.0 * c2 * c0)) / (2.0 * c2);
    else
        nd = 0.5 * h + c0 / c1;
    double d = c / nd + 0.5 * nd * DD;
    if (fabs(nd) < h * 0.01) d = 0.5 * nd * DD;
    return d;
}

// Godunov |grad phi| (levelset2d.cpp:596-610)
__device__ __forceinline__ double godunov(double s0, double dPX, double dMX, double dPY, double dMY) {
    if (s0 >= 0)
        return sqrt(smax(sq(smin(dPX, 0.0)), sq(smax(dMX, 0.0))) + smax(sq(smin(dPY, 0.0)), sq(smax(dMY, 0.0))));
    return sqrt(smax(sq(smax(dPX, 0.0)), sq(smin(dMX, 0.0))) + smax(sq(smax(dPY, 0.0)), sq(smin(dMY, 0.0))));
}

struct LsConst {
    DivH ddx, ddy, ddx2, ddy2;  // /dx, /dy, /(dx*dx), /(dy*dy)
    double dx, dy, eps, adt, thick;
};

// ENO (sub = false) or subcell ENO (sub = true) |grad phi| at interior (i,j).
template <bool SUB>
__device__ __forceinline__ double absgrad(const Grid &g, const LsConst &K, const double *__restrict__ ls,
                                          const double *__restrict__ ls0, int i, int j) {
    double dPX, dMX, dPY, dMY;
    const double c = ls[IX(g, i, j)];
    eno_1d(ls[IX(g, i - 2, j)], ls[IX(g, i - 1, j)], c, ls[IX(g, i + 1, j)], ls[IX(g, i + 2, j)], K.dx, K.ddx, K.ddx2,
           dPX, dMX);
    eno_1d(ls[IX(g, i, j - 2)], ls[IX(g, i, j - 1)], c, ls[IX(g, i, j + 1)], ls[IX(g, i, j + 2)], K.dy, K.ddy, K.ddy2,
           dPY, dMY);
    const double x0 = ls0[IX(g, i, j)];
    if (SUB) {
        const double xm1 = ls0[IX(g, i - 1, j)], xp1 = ls0[IX(g, i + 1, j)];
        if (x0 * xp1 < 0) dPX = subcell_plus(K.dx, K.ddx, K.ddx2, c, xm1, x0, xp1, ls0[IX(g, i + 2, j)]);
        if (x0 * xm1 < 0) dMX = subcell_minus(K.dx, K.ddx, K.ddx2, c, ls0[IX(g, i - 2, j)], xm1, x0, xp1);
        const double ym1 = ls0[IX(g, i, j - 1)], yp1 = ls0[IX(g, i, j + 1)];
        if (x0 * yp1 < 0) dPY = subcell_plus(K.dy, K.ddy, K.ddy2, c, ym1, x0, yp1, ls0[IX(g, i, j + 2)]);
        if (x0 * ym1 < 0) dMY = subcell_minus(K.dy, K.ddy, K.ddy2, c, ls0[IX(g, i, j - 2)], ym1, x0, yp1);
    }
    return godunov(x0, dPX, dMX, dPY, dMY);
}

// GetSussmanReinitConstraint at interior (i,j) (levelset2d.cpp:787-893);
// returns the value added to phi (0 when hd == 0).
__device__ __forceinline__ double sussman_constraint(const Grid &g, const LsConst &K, const double *__restrict__ ls,
                                                     const double *__restrict__ ls0, double hd, int i, int j) {
    if (hd == 0.0) return 0.0;
    const DivH &ddx = K.ddx, &ddy = K.ddy;
#define L_(a, b) ls[IX(g, i + (a), j + (b))]
#define I_(a, b) ls0[IX(g, i + (a), j + (b))]
    double lf[3][3], lif[3][3], dA[3][3];
    lf[0][0] = 0.25 * (L_(0, 0) + L_(-1, 0) + L_(-1, -1) + L_(0, -1));
    lf[0][1] = 0.5 * (L_(0, -1) + L_(0, 0));
    lf[0][2] = 0.25 * (L_(0, 0) + L_(-1, 0) + L_(-1, 1) + L_(0, 1));
    lf[1][0] = 0.5 * (L_(0, -1) + L_(0, 0));
    lf[1][1] = L_(0, 0);
    lf[1][2] = 0.5 * (L_(0, 0) + L_(0, 1));
    lf[2][0] = 0.25 * (L_(0, 0) + L_(1, 0) + L_(1, -1) + L_(0, -1));
    lf[2][1] = 0.5 * (L_(0, 0) + L_(1, 0));
    lf[2][2] = 0.25 * (L_(0, 0) + L_(1, 0) + L_(1, 1) + L_(0, 1));
    lif[0][0] = 0.25 * (I_(0, 0) + I_(-1, 0) + I_(-1, -1) + I_(0, -1));
    lif[0][1] = 0.5 * (I_(0, -1) + I_(0, 0));
    lif[0][2] = 0.25 * (I_(0, 0) + I_(-1, 0) + I_(-1, 1) + I_(0, 1));
    lif[1][0] = 0.5 * (I_(0, -1) + I_(0, 0));
    lif[1][1] = I_(0, 0);
    lif[1][2] = 0.5 * (I_(0, 0) + I_(0, 1));
    lif[2][0] = 0.25 * (I_(0, 0) + I_(1, 0) + I_(1, -1) + I_(0, -1));
    lif[2][1] = 0.5 * (I_(0, 0) + I_(1, 0));
    lif[2][2] = 0.25 * (I_(0, 0) + I_(1, 0) + I_(1, 1) + I_(0, 1));
    dA[0][0] = sqrt(sq(ddx((I_(0, 0) + I_(0, -1)) * 0.5 - 0.5 * (I_(-1, 0) + I_(-1, -1)))) +
                    sq(ddy(lif[0][1] - 0.5 * (I_(0, -1) + I_(-1, -1)))));
    dA[0][1] = sqrt(sq(ddx(lif[1][1] - I_(-1, 0))) + sq(ddy(lif[2][0] - lif[0][0])));
    dA[0][2] = sqrt(sq(ddx(lif[1][2] - -0.5 * (I_(-1, 0) + I_(-1, 1)))) + sq(ddy(0.5 * (I_(-1, 1) + I_(0, 1)) - lif[0][1])));
    dA[1][0] = sqrt(sq(ddx(lif[2][0] - lif[0][0])) + sq(ddy(lif[1][1] - 0.5 * (I_(0, -1) + I_(0, 0)))));
    dA[1][1] = sqrt(sq(ddx(lif[2][1] - lif[0][1])) + sq(ddy(lif[1][2] - lif[1][0])));
    dA[1][2] = sqrt(sq(ddx(lif[2][2] - lif[0][2])) + sq(ddy(I_(0, 1) - lif[1][1])));
    dA[2][0] = sqrt(sq(ddx(0.5 * (I_(1, 0) + I_(1, -1)) - lif[1][0])) + sq(ddy(lif[2][1] - 0.5 * (I_(0, -1) + I_(1, -1)))));
    dA[2][1] = sqrt(sq((I_(1, 0) - lif[1][1]) / (2.0 * K.dx)) + sq(ddy(lif[2][2] - lif[2][0])));
    dA[2][2] = sqrt(sq(ddx(0.5 * (I_(1, 0) + I_(1, 1)) - lif[1][1])) + sq(ddy(0.5 * (I_(0, 1) + I_(1, 1)) - lif[2][1])));
#undef L_
#undef I_
    double s1 = 0.0, s2 = 0.0, f11 = 0.0, Hp11 = 0.0, L11 = 0.0;
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) {
            const double Hp = fabs(lf[a][b]) > K.thick ? 0.0 : 0.5 / K.eps + 0.5 / K.eps * cos(kPi * lf[a][b] / K.eps);
            const double L = (lf[a][b] - lif[a][b]) / K.adt;
            const double f = Hp * dA[a][b];
            s1 += Hp * L;
            s2 += Hp * f;
            if (a == 1 && b == 1) { f11 = f; Hp11 = Hp; L11 = L; }
        }
    s1 += 15.0 * Hp11 * L11;
    s2 += 15.0 * Hp11 * f11;
    return 0.0 - K.adt * f11 * s1 / s2;
}

// UpdateHeavisideFuncDeriv at one value (levelset2d.cpp:27-41)
__device__ __forceinline__ double heaviside_deriv(double l, double eps) {
    return fabs(l) > eps ? 0.0 : 0.5 * (1.0 / eps + cos(kPi * l / eps));
}

// GetSmoothedSignFunc at one value (:914-923)
__device__ __forceinline__ double smoothed_sign(double l, double eps) { return l / sqrt(l * l + eps * eps); }

}  // namespace asd2g
