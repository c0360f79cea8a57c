/*
 * count_ops.cpp -- counts the floating-point operations of one cell-stage
 * by running the oracle's face pipeline (oracle_core.h) with an
 * operation-counting number type.  TEST INFRASTRUCTURE: built by
 * `make -C oracle` into oracle/count_ops; its output pins the constant the
 * benchmark uses for the FP32 compute roofline (tests/test_oracle.py).
 *
 * Counting rule: add, sub, mul, div, sqrt, compare, min, max, abs = 1 each
 * (a fused multiply-add would count 2 = one mul + one add; the oracle has
 * none, so this is the same count).  Conversions are free.
 *
 * One cell-stage of the fused kernel evaluates:
 *   3 faces (its left x, y and z face; boundary extra faces amortise to 0)
 *     each = face_flux minus the primitive conversion of its 6 stencil
 *     cells (the kernel converts each cell once, not at every face);
 *   1 primitive conversion of the cell itself;
 *   the divergence, extra terms, register and state update of the cell.
 * Output: one line "flops_per_cell_stage <n> face <f> prim <p> cell <c>".
 */
#include <cmath>
#include <cstdio>
#include <cstdlib>

struct CF;
static long long g_ops = 0;

struct CF
{
    double v;
    CF() : v(0) {}
    CF(double x) : v(x) {}
    CF& operator+=(const CF& o) { ++g_ops; v += o.v; return *this; }
    CF& operator-=(const CF& o) { ++g_ops; v -= o.v; return *this; }
    CF& operator*=(const CF& o) { ++g_ops; v *= o.v; return *this; }
    CF& operator/=(const CF& o) { ++g_ops; v /= o.v; return *this; }
    CF operator-() const { return CF(-v); }   /* sign flip: free */
    explicit operator double() const { return v; }
};
/* host-side dt arithmetic of the oracle's step() (not part of a cell-stage) */
static inline double operator/(double a, const CF& b) { ++g_ops; return a / b.v; }
static inline CF operator+(const CF& a, const CF& b) { ++g_ops; return CF(a.v + b.v); }
static inline CF operator-(const CF& a, const CF& b) { ++g_ops; return CF(a.v - b.v); }
static inline CF operator*(const CF& a, const CF& b) { ++g_ops; return CF(a.v * b.v); }
static inline CF operator/(const CF& a, const CF& b) { ++g_ops; return CF(a.v / b.v); }
static inline bool operator==(const CF& a, const CF& b) { ++g_ops; return a.v == b.v; }
static inline bool operator<(const CF& a, const CF& b) { ++g_ops; return a.v < b.v; }
static inline CF cf_min(const CF& a, const CF& b) { ++g_ops; return CF(a.v < b.v ? a.v : b.v); }
static inline CF cf_max(const CF& a, const CF& b) { ++g_ops; return CF(a.v > b.v ? a.v : b.v); }
static inline CF cf_sqrt(const CF& a) { ++g_ops; return CF(std::sqrt(a.v)); }
static inline CF cf_abs(const CF& a) { ++g_ops; return CF(std::fabs(a.v)); }

#define ORACLE_WENOEPS 1e-6
/* the operation count is the WENO5 build's */
static int g_oracle_weno3 = 0;
#define REAL CF
#define SFX(name) name##_cnt
#define RMIN cf_min
#define RMAX cf_max
#define RSQRT cf_sqrt
#define RABS cf_abs
#pragma GCC diagnostic ignored "-Wunknown-pragmas"
#include "oracle_core.h"

int main()
{
    /* a representative liquid stencil (the count does not depend on values
     * except through the sign of s*, which changes no operation count) */
    CF s[7][6];
    for (int j = 0; j < 6; ++j)
    {
        s[0][j] = CF(1000.0 + j);
        s[1][j] = CF(1e-3 * j);
        s[2][j] = CF(-2e-3 * j);
        s[3][j] = CF(5e-4);
        s[4][j] = CF(4846.8 + 0.1 * j);
        s[5][j] = CF(1.0 / 5.59);
        s[6][j] = CF(6.59 * 4096.0 / 5.59);
    }
    CF out[12];
    g_ops = 0;
    face_flux_cnt(s, 0, out);
    const long long face_total = g_ops;

    /* primitive conversion of one cell, as face_flux does it per stencil cell */
    CF r(1000.0), u(1.0), v(2.0), w(3.0), e(4846.8), G(0.1789), P(4828.9);
    g_ops = 0;
    u /= r; v /= r; w /= r;
    CF p = (e - 0.5f*r*(u*u + v*v + w*w) - P) / G;
    (void)p;
    const long long prim = g_ops;

    /* extra terms, divergence, register and state update of one cell
     * (oracle_core.h stage(): the per-cell loop and the update loop) */
    CF f[6][12];
    for (int a = 0; a < 6; ++a) for (int b = 0; b < 12; ++b) f[a][b] = CF(1.0 + a + 0.01 * b);
    CF R7[7], U7[7], rhs[7];
    for (int k = 0; k < 7; ++k) { R7[k] = CF(0.1 * k); U7[k] = CF(1.0 + k); }
    const CF a(-17.0 / 32), b(8.0 / 9), dtinvh(0.057), factor6(1.0f / 6.0f);
    g_ops = 0;
    CF sumG = f[0][8] + f[1][7];
    CF sumP = f[0][10] + f[1][9];
    CF divU = f[1][11] - f[0][11];
    sumG += f[2][8] + f[3][7];
    sumP += f[2][10] + f[3][9];
    divU += f[3][11] - f[2][11];
    sumG += f[4][8] + f[5][7];
    sumP += f[4][10] + f[5][9];
    divU += f[5][11] - f[4][11];
    for (int k = 0; k < 7; ++k)
    {
        const CF fxp = f[1][k], fxm = f[0][k], fyp = f[3][k], fym = f[2][k], fzp = f[5][k], fzm = f[4][k];
        CF rk;
        if (k == 5)      rk = dtinvh*(fxp - fxm + fyp - fym + fzp - fzm - divU * sumG * factor6);
        else if (k == 6) rk = dtinvh*(fxp - fxm + fyp - fym + fzp - fzm - divU * sumP * factor6);
        else             rk = dtinvh*(fxp - fxm + fyp - fym + fzp - fzm);
        rhs[k] = a*R7[k] - rk;
        U7[k] = b*rhs[k] + U7[k];
    }
    const long long cell = g_ops;

    const long long face_core = face_total - 6 * prim;
    const long long per_cell = 3 * face_core + prim + cell;
    std::printf("flops_per_cell_stage %lld face %lld face_core %lld prim %lld cell %lld\n",
                per_cell, face_total, face_core, prim, cell);
    return 0;
}
