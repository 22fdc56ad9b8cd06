// Per-cell arithmetic of the level-set and momentum stencils, in the
// reference's operation order, templated on the element type T.  With
// T = double and -fmad=false (no product fused into an add) every +, -, *, /
// and sqrt below rounds exactly as the reference's x86-64 build does, which
// makes the FP64 results bit-identical to the reference wherever no
// cos/sin/pow(x,3) is involved; every literal is written T(<literal>), which
// is the same double constant.  T = float is the mixed-precision path.
#pragma once
#include "internal.cuh"

namespace asd2g {

constexpr double kPi = 3.14159265358979323846;  // the value of M_PI

template <typename T> __device__ __forceinline__ T sq(T x) { return x * x; }
template <typename T> __device__ __forceinline__ int isgn(T v) { return (v > 0) - (v < 0); }
// std::max / std::min semantics
template <typename T> __device__ __forceinline__ T smax(T a, T b) { return (a < b) ? b : a; }
template <typename T> __device__ __forceinline__ T smin(T a, T b) { return (b < a) ? b : a; }

template <typename T> __device__ __forceinline__ T quiet_nan();
template <> __device__ __forceinline__ double quiet_nan<double>() { return __longlong_as_double(0x7ff8000000000000ULL); }
template <> __device__ __forceinline__ float quiet_nan<float>() { return __int_as_float(0x7fc00000); }

// LevelSetSolver2D::MinMod, levelset2d.cpp:1036-1046
template <typename T> __device__ __forceinline__ T minmod(T a, T b) {
    const T p = a * b;
    if ((fabs(a) <= fabs(b)) && (p > 0)) return a;
    if ((fabs(a) > fabs(b)) && (p > 0)) return b;
    if (p <= 0) return T(0.0);
    return quiet_nan<T>();
}

// Jiang-Peng weights (0.1, 0.6, 0.3) / (eps + IS)^2, normalised.  FP64: the
// reference's divisions as written.  FP32 (not bit-exact by design): the
// fast single-precision divide for the three alphas and one reciprocal of
// their sum -- the weights are a smoothness heuristic, and these divisions
// were a third of the FP32 stencil's instructions.
template <typename T> __device__ __forceinline__ void weno_weights(T is0, T is1, T is2, T eps, T &w0, T &w1, T &w2) {
    if constexpr (sizeof(T) == sizeof(float)) {
        const float a0 = __fdividef(0.1f, sq(eps + is0)), a1 = __fdividef(0.6f, sq(eps + is1)),
                    a2 = __fdividef(0.3f, sq(eps + is2));
        const float r = __fdividef(1.0f, a0 + a1 + a2);
        w0 = a0 * r;
        w1 = a1 * r;
        w2 = a2 * r;
    } else {
        const T a0 = T(0.1) / sq(eps + is0), a1 = T(0.6) / sq(eps + is1), a2 = T(0.3) / sq(eps + is2);
        w0 = a0 / (a0 + a1 + a2);
        w1 = a1 / (a0 + a1 + a2);
        w2 = a2 / (a0 + a1 + a2);
    }
}

// UnitHJWENO5 at one point (levelset2d.cpp:159-262).  D[k] = DFPlus[i-3+k],
// k = 0..5.  dv divides by the spacing d.
template <typename T>
__device__ __forceinline__ void weno5_point(const T D[6], const DivHT<T> &dv, T &FP, T &FM) {
    const T eps = T(1e-6);
    // phi^- uses DFPlus[i-3 .. i+1]
    {
        const T d3 = D[0], d2 = D[1], d1 = D[2], d0 = D[3], p1 = D[4];
        const T is0 = T(13.0 / 12.0) * sq(dv(d3 - T(2.0) * d2 + d1)) + T(1.0 / 4.0) * sq(dv(d3 - T(4.0) * d2 + T(3.0) * d1));
        const T is1 = T(13.0 / 12.0) * sq(dv(d2 - T(2.0) * d1 + d0)) + T(1.0 / 4.0) * sq(dv(d2 - d0));
        const T is2 = T(13.0 / 12.0) * sq(dv(d1 - T(2.0) * d0 + p1)) + T(1.0 / 4.0) * sq(dv(T(3.0) * d1 - T(4.0) * d0 + p1));
        T w0, w1, w2;
        weno_weights(is0, is1, is2, eps, w0, w1, w2);
        FM = dv(w0 * (T(1.0 / 3.0) * d3 - T(7.0 / 6.0) * d2 + T(11.0 / 6.0) * d1)) +
             dv(w1 * (T(-1.0 / 6.0) * d2 + T(5.0 / 6.0) * d1 + T(1.0 / 3.0) * d0)) +
             dv(w2 * (T(1.0 / 3.0) * d1 + T(5.0 / 6.0) * d0 - T(1.0 / 6.0) * p1));
    }
    // phi^+ uses DFPlus[i-2 .. i+2]
    {
        const T m2 = D[1], m1 = D[2], d0 = D[3], p1 = D[4], p2 = D[5];
        const T is0 = T(13.0 / 12.0) * sq(dv(p2 - T(2.0) * p1 + d0)) + T(1.0 / 4.0) * sq(dv(p2 - T(4.0) * p1 + T(3.0) * d0));
        const T is1 = T(13.0 / 12.0) * sq(dv(p1 - T(2.0) * d0 + m1)) + T(1.0 / 4.0) * sq(dv(p1 - m1));
        const T is2 = T(13.0 / 12.0) * sq(dv(d0 - T(2.0) * m1 + m2)) + T(1.0 / 4.0) * sq(dv(T(3.0) * d0 - T(4.0) * m1 + m2));
        T w0, w1, w2;
        weno_weights(is0, is1, is2, eps, w0, w1, w2);
        FP = dv(w0 * (T(1.0 / 3.0) * p2 - T(7.0 / 6.0) * p1 + T(11.0 / 6.0) * d0)) +
             dv(w1 * (T(-1.0 / 6.0) * p1 + T(5.0 / 6.0) * d0 + T(1.0 / 3.0) * m1)) +
             dv(w2 * (T(1.0 / 3.0) * d0 + T(5.0 / 6.0) * m1 - T(1.0 / 6.0) * m2));
    }
}

// Signed-velocity blend (HJWENO5_LS_2D :144-154; AddConvectionFU :367-371).
template <typename T>
__device__ __forceinline__ T weno_blend(T xp, T xm, T yp, T ym, T ax, T ay) {
    return T(0.5) * (xp + xm) + T(0.5) * (yp + ym) - ax * (T(0.5) * (xp - xm)) - ay * (T(0.5) * (yp - ym));
}

// Second-order ENO one-sided differences along one axis from five values
// c[-2..2] (ENO_DerivAbsLS_2D :567-594).  dh divides by h, dh2 by h*h.
template <typename T>
__device__ __forceinline__ void eno_1d(T lm2, T lm1, T l0, T lp1, T lp2, T h, const DivHT<T> &dh, const DivHT<T> &dh2,
                                       T &dP, T &dM) {
    dP = dh(lp1 - l0) - h * T(0.5) * minmod(dh2(lm1 - T(2.0) * l0 + lp1), dh2(l0 - T(2.0) * lp1 + lp2));
    dM = dh(l0 - lm1) + h * T(0.5) * minmod(dh2(lm1 - T(2.0) * l0 + lp1), dh2(lm2 - T(2.0) * lm1 + l0));
}

// Root (-c1 + sg * sqrt(c1^2 - 4 c2 c0)) / (2 c2) of c2 x^2 + c1 x + c0 (sg =
// +-1).  FP64 evaluates it as written, which is the reference's rounding.
// In FP32 that form cancels when -c1 and the square root have opposite
// signs and c2 is small (an error of ~1e-4 in phi after one reinitialisation
// of an exact distance function); there the same root is taken from the
// product of the roots, 2 c0 / (-c1 - sg * sqrt(...)), which does not cancel.
template <typename T> __device__ __forceinline__ T quad_root(T c2, T c1, T c0, T sg) {
    const T sd = sg * sqrt(c1 * c1 - T(4.0) * c2 * c0);
    if constexpr (sizeof(T) == sizeof(float)) {
        if ((-c1) * sd < T(0.0)) return (T(2.0) * c0) / (-c1 - sd);
    }
    return (-c1 + sd) / (T(2.0) * c2);
}

// Min-Gibou subcell derivative at a cell whose + neighbour changes sign in
// phi0 (levelset2d.cpp:655-681).  c = phi at the cell; i0m1..i0p2 = phi0.
template <typename T>
__device__ __forceinline__ T subcell_plus(T h, const DivHT<T> &dh, const DivHT<T> &dh2, T c, T i0m1, T i00, T i0p1,
                                          T i0p2) {
    const T DD = minmod(dh2(i0m1 - T(2.0) * i00 + i0p1), dh2(i00 - T(2.0) * i0p1 + i0p2));
    const T c2 = T(0.5) * DD;
    const T c1 = dh(i0p1 - i00);
    const T c0 = (i0p1 + i00) * T(0.5) - c2 * h * h * T(0.25);
    T nd;
    if (fabs(c2) > T(1.0e-10))
        nd = T(0.5) * h + quad_root(c2, c1, c0, T(-isgn(i00)));
    else
        nd = T(0.5) * h - c0 / c1;
    T d = -c / nd - T(0.5) * nd * DD;
    if (fabs(nd) < h * T(0.01)) d = T(-0.5) * nd * DD;
    return d;
}

// ... and at a cell whose - neighbour changes sign (:686-711).
template <typename T>
__device__ __forceinline__ T subcell_minus(T h, const DivHT<T> &dh, const DivHT<T> &dh2, T c, T i0m2, T i0m1, T i00,
                                           T i0p1) {
    const T DD = minmod(dh2(i0m1 - T(2.0) * i00 + i0p1), dh2(i0m2 - T(2.0) * i0m1 + i00));
    const T c2 = T(0.5) * DD;
    const T c1 = dh(i00 - i0m1);
    const T c0 = (i00 + i0m1) * T(0.5) - c2 * h * h * T(0.25);
    T nd;
    if (fabs(c2) > T(1.0e-10))
        nd = T(0.5) * h - quad_root(c2, c1, c0, T(isgn(i00)));
    else
        nd = T(0.5) * h + c0 / c1;
    T d = c / nd + T(0.5) * nd * DD;
    if (fabs(nd) < h * T(0.01)) d = T(0.5) * nd * DD;
    return d;
}

// Godunov |grad phi| (levelset2d.cpp:596-610)
template <typename T>
__device__ __forceinline__ T godunov(T s0, T dPX, T dMX, T dPY, T dMY) {
    const T z = T(0.0);
    if (s0 >= 0) return sqrt(smax(sq(smin(dPX, z)), sq(smax(dMX, z))) + smax(sq(smin(dPY, z)), sq(smax(dMY, z))));
    return sqrt(smax(sq(smax(dPX, z)), sq(smin(dMX, z))) + smax(sq(smax(dPY, z)), sq(smin(dMY, z))));
}

template <typename T>
struct LsConstT {
    DivHT<T> ddx, ddy, ddx2, ddy2;  // /dx, /dy, /(dx*dx), /(dy*dy)
    T dx, dy, eps, adt, thick;
};
using LsConst = LsConstT<double>;

// ENO (sub = false) or subcell ENO (sub = true) |grad phi| at interior (i,j).
template <bool SUB, typename T>
__device__ __forceinline__ T absgrad(const Grid &g, const LsConstT<T> &K, const T *__restrict__ ls,
                                     const T *__restrict__ ls0, int i, int j) {
    T dPX, dMX, dPY, dMY;
    const T c = ls[IX(g, i, j)];
    eno_1d(ls[IX(g, i - 2, j)], ls[IX(g, i - 1, j)], c, ls[IX(g, i + 1, j)], ls[IX(g, i + 2, j)], K.dx, K.ddx, K.ddx2,
           dPX, dMX);
    eno_1d(ls[IX(g, i, j - 2)], ls[IX(g, i, j - 1)], c, ls[IX(g, i, j + 1)], ls[IX(g, i, j + 2)], K.dy, K.ddy, K.ddy2,
           dPY, dMY);
    const T x0 = ls0[IX(g, i, j)];
    if (SUB) {
        const T xm1 = ls0[IX(g, i - 1, j)], xp1 = ls0[IX(g, i + 1, j)];
        if (x0 * xp1 < 0) dPX = subcell_plus(K.dx, K.ddx, K.ddx2, c, xm1, x0, xp1, ls0[IX(g, i + 2, j)]);
        if (x0 * xm1 < 0) dMX = subcell_minus(K.dx, K.ddx, K.ddx2, c, ls0[IX(g, i - 2, j)], xm1, x0, xp1);
        const T ym1 = ls0[IX(g, i, j - 1)], yp1 = ls0[IX(g, i, j + 1)];
        if (x0 * yp1 < 0) dPY = subcell_plus(K.dy, K.ddy, K.ddy2, c, ym1, x0, yp1, ls0[IX(g, i, j + 2)]);
        if (x0 * ym1 < 0) dMY = subcell_minus(K.dy, K.ddy, K.ddy2, c, ls0[IX(g, i, j - 2)], ym1, x0, yp1);
    }
    return godunov(x0, dPX, dMX, dPY, dMY);
}

// GetSussmanReinitConstraint at interior (i,j) (levelset2d.cpp:787-893);
// returns the value added to phi (0 when hd == 0).
template <typename T>
__device__ __forceinline__ T sussman_constraint(const Grid &g, const LsConstT<T> &K, const T *__restrict__ ls,
                                                const T *__restrict__ ls0, T hd, int i, int j) {
    if (hd == T(0.0)) return T(0.0);
    const DivHT<T> &ddx = K.ddx, &ddy = K.ddy;
#define L_(a, b) ls[IX(g, i + (a), j + (b))]
#define I_(a, b) ls0[IX(g, i + (a), j + (b))]
    T lf[3][3], lif[3][3], dA[3][3];
    lf[0][0] = T(0.25) * (L_(0, 0) + L_(-1, 0) + L_(-1, -1) + L_(0, -1));
    lf[0][1] = T(0.5) * (L_(0, -1) + L_(0, 0));
    lf[0][2] = T(0.25) * (L_(0, 0) + L_(-1, 0) + L_(-1, 1) + L_(0, 1));
    lf[1][0] = T(0.5) * (L_(0, -1) + L_(0, 0));
    lf[1][1] = L_(0, 0);
    lf[1][2] = T(0.5) * (L_(0, 0) + L_(0, 1));
    lf[2][0] = T(0.25) * (L_(0, 0) + L_(1, 0) + L_(1, -1) + L_(0, -1));
    lf[2][1] = T(0.5) * (L_(0, 0) + L_(1, 0));
    lf[2][2] = T(0.25) * (L_(0, 0) + L_(1, 0) + L_(1, 1) + L_(0, 1));
    lif[0][0] = T(0.25) * (I_(0, 0) + I_(-1, 0) + I_(-1, -1) + I_(0, -1));
    lif[0][1] = T(0.5) * (I_(0, -1) + I_(0, 0));
    lif[0][2] = T(0.25) * (I_(0, 0) + I_(-1, 0) + I_(-1, 1) + I_(0, 1));
    lif[1][0] = T(0.5) * (I_(0, -1) + I_(0, 0));
    lif[1][1] = I_(0, 0);
    lif[1][2] = T(0.5) * (I_(0, 0) + I_(0, 1));
    lif[2][0] = T(0.25) * (I_(0, 0) + I_(1, 0) + I_(1, -1) + I_(0, -1));
    lif[2][1] = T(0.5) * (I_(0, 0) + I_(1, 0));
    lif[2][2] = T(0.25) * (I_(0, 0) + I_(1, 0) + I_(1, 1) + I_(0, 1));
    dA[0][0] = sqrt(sq(ddx((I_(0, 0) + I_(0, -1)) * T(0.5) - T(0.5) * (I_(-1, 0) + I_(-1, -1)))) +
                    sq(ddy(lif[0][1] - T(0.5) * (I_(0, -1) + I_(-1, -1)))));
    dA[0][1] = sqrt(sq(ddx(lif[1][1] - I_(-1, 0))) + sq(ddy(lif[2][0] - lif[0][0])));
    dA[0][2] = sqrt(sq(ddx(lif[1][2] - T(-0.5) * (I_(-1, 0) + I_(-1, 1)))) + sq(ddy(T(0.5) * (I_(-1, 1) + I_(0, 1)) - lif[0][1])));
    dA[1][0] = sqrt(sq(ddx(lif[2][0] - lif[0][0])) + sq(ddy(lif[1][1] - T(0.5) * (I_(0, -1) + I_(0, 0)))));
    dA[1][1] = sqrt(sq(ddx(lif[2][1] - lif[0][1])) + sq(ddy(lif[1][2] - lif[1][0])));
    dA[1][2] = sqrt(sq(ddx(lif[2][2] - lif[0][2])) + sq(ddy(I_(0, 1) - lif[1][1])));
    dA[2][0] = sqrt(sq(ddx(T(0.5) * (I_(1, 0) + I_(1, -1)) - lif[1][0])) + sq(ddy(lif[2][1] - T(0.5) * (I_(0, -1) + I_(1, -1)))));
    dA[2][1] = sqrt(sq((I_(1, 0) - lif[1][1]) / (T(2.0) * K.dx)) + sq(ddy(lif[2][2] - lif[2][0])));
    dA[2][2] = sqrt(sq(ddx(T(0.5) * (I_(1, 0) + I_(1, 1)) - lif[1][1])) + sq(ddy(T(0.5) * (I_(0, 1) + I_(1, 1)) - lif[2][1])));
#undef L_
#undef I_
    T s1 = T(0.0), s2 = T(0.0), f11 = T(0.0), Hp11 = T(0.0), L11 = T(0.0);
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) {
            const T Hp = fabs(lf[a][b]) > K.thick ? T(0.0) : T(0.5) / K.eps + T(0.5) / K.eps * cos(T(kPi) * lf[a][b] / K.eps);
            const T L = (lf[a][b] - lif[a][b]) / K.adt;
            const T f = Hp * dA[a][b];
            s1 += Hp * L;
            s2 += Hp * f;
            if (a == 1 && b == 1) { f11 = f; Hp11 = Hp; L11 = L; }
        }
    s1 += T(15.0) * Hp11 * L11;
    s2 += T(15.0) * Hp11 * f11;
    return T(0.0) - K.adt * f11 * s1 / s2;
}

// UpdateHeavisideFuncDeriv at one value (levelset2d.cpp:27-41)
template <typename T> __device__ __forceinline__ T heaviside_deriv(T l, T eps) {
    return fabs(l) > eps ? T(0.0) : T(0.5) * (T(1.0) / eps + cos(T(kPi) * l / eps));
}

// GetSmoothedSignFunc at one value (:914-923).  FP32 (the mixed path):
// l * rsqrt(l^2 + eps^2), one MUFU op instead of a divide and a square root.
template <typename T> __device__ __forceinline__ T smoothed_sign(T l, T eps) {
    if constexpr (sizeof(T) == sizeof(float)) return l * rsqrtf(fmaf(l, l, eps * eps));
    else return l / sqrt(l * l + eps * eps);
}

}  // namespace asd2g
