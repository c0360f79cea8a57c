// mpcf_math.cuh -- device math of one cell face: WENO5 reconstruction with
// clipping, Einfeldt / Batten wave speeds and the HLLC fluxes of the
// 7-component stiffened-gas system, written for sm_100a.
//
// The arithmetic follows the reference device functions
//   WENO5-JS             source/GPU/GPUonly.cuh:99-194
//   Einfeldt, s*         source/GPU/GPUonly.cuh:802-866
//   HLLC fluxes          source/GPU/GPUonly.cuh:869-1026
//   extra-term velocity  source/GPU/GPUonly.cuh:1029-1042
// in the same evaluation order.  A precision policy selects the rounding:
//
//   PolRef32   float storage and arithmetic, the reference's double-promoted
//              sub-expressions kept in double, IEEE division and sqrt.  Its
//              translation unit is compiled with --fmad=false, so every
//              operation rounds exactly like the literal C semantics of the
//              reference source: results are bit-identical to the CPU
//              restatement built with -ffp-contract=off.
//   PolFast32  float everywhere; WENO smoothness indicators in factored
//              (cancellation-free, shared-curvature) form, weights from
//              single-precision reciprocals, fused multiply-adds allowed.
//   PolMixed   PolFast32 plus the stiffened-gas pressure recovery in
//              compensated FP32 (two-sum) and FP64 conservation sums.
//   PolFP64    double storage and arithmetic (the all-FP64 GPU oracle run).
//   PolFast64  double storage and arithmetic with the fast forms' algebra
//              (factored indicators and fluxes, refined double reciprocals):
//              the tuned FP64 yardstick of the mixed form.
//   PolRef32W3, PolFP64W3  the two reference-rounding forms with the
//              reference's compile-time WENO3 reconstruction.
//
// Primitive index convention used throughout the device code:
//   0 rho, 1 u, 2 v, 3 w, 4 p, 5 G = 1/(gamma-1), 6 P = gamma*pc/(gamma-1)
// Face output slots: 0..6 fluxes of (rho, rho u, rho v, rho w, E, G, P),
//   7 Gm, 8 Gp, 9 Pm, 10 Pp, 11 u* (extra-term velocity).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace mpcf {

#ifndef MPCF_WENOEPS
#define MPCF_WENOEPS 1e-6   // Makefile.config:15 (weps ?= 1e-6)
#endif

struct PolRef32  { typedef float  T; static constexpr bool kFastWeno = false; static constexpr bool kCompP = false; static constexpr bool kRefRounding = true;  static constexpr bool kWeno3 = false; static constexpr int id = 0; };
struct PolFast32 { typedef float  T; static constexpr bool kFastWeno = true;  static constexpr bool kCompP = false; static constexpr bool kRefRounding = false; static constexpr bool kWeno3 = false; static constexpr int id = 1; };
struct PolMixed  { typedef float  T; static constexpr bool kFastWeno = true;  static constexpr bool kCompP = true;  static constexpr bool kRefRounding = false; static constexpr bool kWeno3 = false; static constexpr int id = 2; };
struct PolFP64   { typedef double T; static constexpr bool kFastWeno = false; static constexpr bool kCompP = false; static constexpr bool kRefRounding = true;  static constexpr bool kWeno3 = false; static constexpr int id = 3; };
struct PolFast64 { typedef double T; static constexpr bool kFastWeno = true;  static constexpr bool kCompP = false; static constexpr bool kRefRounding = false; static constexpr bool kWeno3 = false; static constexpr int id = 4; };
// The reference's compile-time WENO3 build (-D_WENO3_, GPUonly.cuh:102,141)
// of the two reference-rounding forms.
struct PolRef32W3 { typedef float  T; static constexpr bool kFastWeno = false; static constexpr bool kCompP = false; static constexpr bool kRefRounding = true; static constexpr bool kWeno3 = true; static constexpr int id = 0; };
struct PolFP64W3  { typedef double T; static constexpr bool kFastWeno = false; static constexpr bool kCompP = false; static constexpr bool kRefRounding = true; static constexpr bool kWeno3 = true; static constexpr int id = 3; };

__device__ __forceinline__ float  dmin(float a, float b)   { return fminf(a, b); }
__device__ __forceinline__ float  dmax(float a, float b)   { return fmaxf(a, b); }
__device__ __forceinline__ double dmin(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ double dmax(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ float  dsqrt(float a)  { return sqrtf(a); }
__device__ __forceinline__ double dsqrt(double a) { return sqrt(a); }

// Approximate reciprocal of the special-function unit (relative error below
// 2^-22); only the fast policies use it.
__device__ __forceinline__ float rcp_approx(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
// Reciprocal in double precision without a division: the special-function
// unit's approximate reciprocal refined by two Newton-Raphson steps
// y <- y + y (1 - x y) (each step doubles the number of correct bits).
__device__ __forceinline__ double rcp_f64(const double x)
{
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    double e = fma(-x, y, 1.0);
    y = fma(y, e, y);
    e = fma(-x, y, 1.0);
    return fma(y, e, y);
}
// the fast FP64 form's reciprocal
__device__ __forceinline__ double rcp_approx(double x) { return rcp_f64(x); }

// Approximate square root of the special-function unit (fast policies).
__device__ __forceinline__ float sqrt_approx(float x)
{
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// ---------------------------------------------------------------------------
// WENO5 smoothness indicators.  For a window of three consecutive cells
// (x, y, z) left to right, the reference uses three polynomial forms:
//   beta_f(x,y,z) = x(4/3 x - 19/3 y + 11/3 z) + y(25/3 y - 31/3 z) + 10/3 z^2
//   beta_h(x,y,z) = x(4/3 x - 13/3 y +  5/3 z) + y(13/3 y - 13/3 z) +  4/3 z^2
//   beta_g(x,y,z) = x(10/3 x - 31/3 y + 11/3 z) + y(25/3 y - 19/3 z) + 4/3 z^2
// minus side (a..e): is0 = f(a,b,c), is1 = h(b,c,d), is2 = g(c,d,e)
// plus side  (b..f): is0 = g(d,e,f), is1 = h(c,d,e), is2 = f(b,c,d)
// (GPUonly.cuh:102-104 and :141-143, same operation order).
// ---------------------------------------------------------------------------
template <class T> __device__ __forceinline__ T beta_f(const T x, const T y, const T z)
{
    return x*(x*(T)(4./3.)  - y*(T)(19./3.) + z*(T)(11./3.)) + y*(y*(T)(25./3.) - z*(T)(31./3.)) + z*z*(T)(10./3.);
}
template <class T> __device__ __forceinline__ T beta_h(const T x, const T y, const T z)
{
    return x*(x*(T)(4./3.)  - y*(T)(13./3.) + z*(T)(5./3.))  + y*(y*(T)(13./3.) - z*(T)(13./3.)) + z*z*(T)(4./3.);
}
template <class T> __device__ __forceinline__ T beta_g(const T x, const T y, const T z)
{
    return x*(x*(T)(10./3.) - y*(T)(31./3.) + z*(T)(11./3.)) + y*(y*(T)(25./3.) - z*(T)(19./3.)) + z*z*(T)(4./3.);
}

// Both edge values of one cell in the reference-rounding policies, from the
// cells y0..y4 = l-2..l+2 (GPUonly.cuh:99-194):
//   R, the minus side of face l+1/2: indicators (is0, is1, is2) =
//     (beta_f(y0,y1,y2), beta_h(y1,y2,y3), beta_g(y2,y3,y4)), candidates
//     from y0..y4, clipped to [min, max] of y1, y2, y3;
//   L, the plus side of face l-1/2: indicators (beta_g(y2,y3,y4),
//     beta_h(y1,y2,y3), beta_f(y0,y1,y2)), the mirrored candidates, the same
//     clip;
//   weights alpha_j = c_j * (1/(10.0*(is_j+eps)^2)) with c = (1, 6, 3) (the
//   10.0 literal promotes the reciprocal to double, GPUonly.cuh:111-113),
//   w0 = alpha0/sum, w1 = alpha1/sum, w2 = 1 - w0 - w1.
// The reference evaluates each face's two sides separately; the three
// indicator calls, their double reciprocals and the clip bounds of the two
// edges of a cell are the same operations on the same values, so they are
// evaluated once here.  Every other operation is the reference's in its
// order, so R and L are bit-identical to its per-face results.
template <class Pol>
__device__ __forceinline__ void weno_cell_ref(const typename Pol::T y0, const typename Pol::T y1,
        const typename Pol::T y2, const typename Pol::T y3, const typename Pol::T y4,
        typename Pol::T& R, typename Pol::T& L)
{
    typedef typename Pol::T T;
    static_assert(!Pol::kFastWeno, "reference-rounding policies only");
    const T pf = beta_f<T>(y0, y1, y2) + (T)MPCF_WENOEPS;
    const T ph = beta_h<T>(y1, y2, y3) + (T)MPCF_WENOEPS;
    const T pg = beta_g<T>(y2, y3, y4) + (T)MPCF_WENOEPS;
    // the 10.0 literal promotes these to double (GPUonly.cuh:111-113)
    const double qf = ((T)1)/(10.0*pf*pf);
    const double qh = ((T)1)/(10.0*ph*ph);
    const double qg = ((T)1)/(10.0*pg*pg);
    const T a1 = (T)((T)(6)*qh);
    const T lo = dmin(dmin(y1, y2), y3);
    const T hi = dmax(dmax(y1, y2), y3);
    {
        // minus side: indicators (f, h, g)
        const T a0 = (T)((T)(1)*qf), a2 = (T)((T)(3)*qg);
        const T inv = ((T)1)/(a0 + a1 + a2);
        const T w0 = a0 * inv, w1 = a1 * inv, w2 = 1 - w0 - w1;
        const T r = w0*((T)(1.0/3.)*y0-(T)(7./6.)*y1+(T)(11./6.)*y2) + w1*(-(T)(1./6.)*y1+(T)(5./6.)*y2+(T)(1./3.)*y3) + w2*((T)(1./3.)*y2+(T)(5./6.)*y3-(T)(1./6.)*y4);
        R = dmin(dmax(r, lo), hi);
    }
    {
        // plus side: indicators (g, h, f)
        const T a0 = (T)((T)(1)*qg), a2 = (T)((T)(3)*qf);
        const T inv = ((T)1)/(a0 + a1 + a2);
        const T w0 = a0 * inv, w1 = a1 * inv, w2 = 1 - w0 - w1;
        const T r = w0*((T)(1./3.)*y4-(T)(7./6.)*y3+(T)(11./6.)*y2) + w1*(-(T)(1./6.)*y3+(T)(5./6.)*y2+(T)(1./3.)*y1) + w2*((T)(1./3.)*y2+(T)(5./6.)*y1-(T)(1./6.)*y0);
        L = dmin(dmax(r, lo), hi);
    }
}

// ---------------------------------------------------------------------------
// Packed single-precision pairs.  sm_100 executes fma / add / mul on two
// FP32 lanes in one instruction (round-to-nearest per lane, the same result
// as two scalar instructions).  The face pipeline is bound by instruction
// issue, so every left/right-symmetric computation runs as one pair.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 f2(const float a, const float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 f2s(const float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(const float2 a, const float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(const float2 a, const float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 mul2(const float2 a, const float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(const float2 a, const float2 b, const float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 rcp2(const float2 a) { return make_float2(rcp_approx(a.x), rcp_approx(a.y)); }
// HLLC upwind blend w.x * F.x + w.y * F.y of a (left, right) flux pair
__device__ __forceinline__ float blend2(const float2 w, const float2 F) { const float2 t = mul2(F, w); return t.x + t.y; }
// The same pair operations in double precision (the fast FP64 form), lane
// by lane: there are no packed FP64 instructions.
__device__ __forceinline__ double2 f2(const double a, const double b) { return make_double2(a, b); }
__device__ __forceinline__ double2 f2s(const double a) { return make_double2(a, a); }
__device__ __forceinline__ double2 add2(const double2 a, const double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 sub2(const double2 a, const double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 mul2(const double2 a, const double2 b) { return make_double2(a.x * b.x, a.y * b.y); }
__device__ __forceinline__ double2 fma2(const double2 a, const double2 b, const double2 c) { return make_double2(fma(a.x, b.x, c.x), fma(a.y, b.y, c.y)); }
__device__ __forceinline__ double2 rcp2(const double2 a) { return make_double2(rcp_f64(a.x), rcp_f64(a.y)); }
__device__ __forceinline__ double blend2(const double2 w, const double2 F) { const double2 t = mul2(F, w); return t.x + t.y; }
// the pair type of a value type
template <class T> struct PairOf;
template <> struct PairOf<float>  { typedef float2 V; };
template <> struct PairOf<double> { typedef double2 V; };

// Minimum / maximum of three values in one operation (sm_100).
__device__ __forceinline__ float min3f(const float a, const float b, const float c)
{
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float max3f(const float a, const float b, const float c)
{
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ double min3f(const double a, const double b, const double c) { return fmin(fmin(a, b), c); }
__device__ __forceinline__ double max3f(const double a, const double b, const double c) { return fmax(fmax(a, b), c); }

// Both edge values of one cell (fast policies), from the cell and its two
// neighbours on either side, y0..y4 = cells l-2..l+2:
//   R = value at the right edge l+1/2 (minus side of that face),
//   L = value at the left edge l-1/2 (plus side of that face).
// The Jiang-Shu smoothness indicators of the three sub-stencils
// (l-2..l, l-1..l+1, l..l+2) integrate over cell l, so they are the same for
// both edges (GPUonly.cuh:99-194 evaluates them again for every face): with
//   k_j = y_j - 2 y_{j+1} + y_{j+2},  a_0 = y0-4y1+3y2, a_1 = y1-y3,
//   a_2 = 3y2-4y3+y4,  g_j = 1/(13/3 k_j^2 + a_j^2 + 4 eps)^2
// (the indicators times 12/3, a common factor that cancels), the two edges
// weigh them with mirrored linear weights d = (1, 6, 3):
//   R = (y2+y3)/2 - k1/6 + (g0 (k0-k1)/3 + g2 (k1-k2)/2) / (g0 + 6 g1 + 3 g2)
//   L = (y2+y1)/2 - k1/6 - (g2 (k1-k2)/3 + g0 (k0-k1)/2) / (3 g0 + 6 g1 + g2)
// and both are clipped to [min, max] of y1, y2, y3.  Lane x of every pair
// is the right edge, lane y the left edge.
// The same algebra serves the fast FP64 form (T = double, lane by lane).
template <class T>
__device__ __forceinline__ void weno_cell_packed(const T y0, const T y1, const T y2,
                                                 const T y3, const T y4, T& R, T& L)
{
    typedef typename PairOf<T>::V V;
    constexpr T e4 = (T)(4.0 * MPCF_WENOEPS);
    const V Y04 = f2(y0, y4), Y13 = f2(y1, y3), Y22 = f2s(y2);
    const V K02 = fma2(Y13, f2s((T)-2), add2(Y04, Y22));                        // (k0, k2)
    const T k1  = fma(y2, (T)-2, y1 + y3);
    const V A02 = fma2(Y22, f2s((T)3), fma2(Y13, f2s((T)-4), Y04));             // (a0, a2)
    const T a1  = y1 - y3;
    const V J02 = fma2(mul2(K02, f2s((T)13 / (T)3)), K02, fma2(A02, A02, f2s(e4)));
    const T j1  = fma(k1 * ((T)13 / (T)3), k1, fma(a1, a1, e4));
    const V G02 = rcp2(mul2(J02, J02));                                         // (g0, g2)
    const T g1  = rcp_approx(j1 * j1);
    const V den = fma2(f2(G02.y, G02.x), f2s((T)3), fma2(f2s(g1), f2s((T)6), G02));
    const V E   = mul2(G02, f2(K02.x - k1, k1 - K02.y));                        // (g0 D0, g2 D2)
    const V num = fma2(E, f2((T)1 / (T)3, -(T)1 / (T)3), mul2(f2(E.y, E.x), f2((T)0.5, (T)-0.5)));
    const V p1  = fma2(f2s(k1), f2s(-(T)1 / (T)6), mul2(add2(Y22, f2(y3, y1)), f2s((T)0.5)));
    const V r   = fma2(num, rcp2(den), p1);
    const T lo = min3f(y1, y2, y3), hi = max3f(y1, y2, y3);
    R = dmin(dmax(r.x, lo), hi);
    L = dmin(dmax(r.y, lo), hi);
}

// ---------------------------------------------------------------------------
// HLLC pieces.  sign_star in {-1,0,1}; the two weights (1+s)/2 and (1-s)/2.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int sign_star_of(const float ss)  { return ss == 0 ? 0 : (ss < 0 ? -1 : 1); }
__device__ __forceinline__ int sign_star_of(const double ss) { return ss == 0 ? 0 : (ss < 0 ? -1 : 1); }

// (0.5f*(1+s))*L + (0.5*(1-s))*R.  In the FP32 reference the second weight
// of _hllc_rho is a double literal (GPUonly.cuh:900), which promotes that
// sum to double; kept exactly under the reference rounding policy.
template <class Pol, bool kDoubleSecondWeight>
__device__ __forceinline__ typename Pol::T hllc_blend(const int s, const typename Pol::T L, const typename Pol::T R)
{
    typedef typename Pol::T T;
    if (kDoubleSecondWeight && Pol::kRefRounding)
        return (T)((double)((0.5f*(1 + s)) * L) + (0.5*(1 - s)) * (double)R);
    else
        return (T)(0.5f*(1 + s)) * L + (T)(0.5f*(1 - s)) * R;
}

// Everything one face produces.
template <class T>
struct FaceOut
{
    T f[7];      // fluxes rho, rho u, rho v, rho w, E, G, P
    T Gm, Gp, Pm, Pp, vel;
};

// The face state after reconstruction: m = left (minus), p = right (plus).
// n = normal velocity, t1/t2 = the transverse velocities in the order the
// reference passes them to _hllc_e (x: v,w; y: u,w; z: u,v).
template <class T>
struct FaceState
{
    T rm, rp, nm, np, t1m, t1p, t2m, t2p, pm, pp, Gm, Gp, Pm, Pp;
};

// Wave speeds + HLLC fluxes of one face (GPUkernels.cu:255-289 for x,
// :636-668 for y, :932-963 for z; GPUonly.cuh:802-1042).  `dir` is a runtime
// value: the normal / transverse momenta are scattered with selects, so one
// instance of this code serves all three directions (the face pipeline is
// ~1000 instructions; one copy keeps it resident in the instruction cache).
template <class Pol>
__device__ __forceinline__ void hllc_face(const FaceState<typename Pol::T>& S, const int dir, FaceOut<typename Pol::T>& o)
{
    typedef typename Pol::T T;
    const T rm = S.rm, rp = S.rp, um = S.nm, up = S.np;
    const T pm = S.pm, pp = S.pp, Gm = S.Gm, Gp = S.Gp, Pm = S.Pm, Pp = S.Pp;

    // Einfeldt bounds (GPUonly.cuh:802-847)
    const T Rr   = dsqrt(rp / rm);
    const T Rinv = (T)1.0f / ((T)1.0f + Rr);
    const T cm2 = ((pm + Pm)/Gm + pm) / rm;
    const T cp2 = ((pp + Pp)/Gp + pp) / rp;
    const T cm  = dsqrt(cm2);
    const T cp  = dsqrt(cp2);
    const T eta_2 = (T)0.5f*Rr*Rinv*Rinv;
    const T d2    = (cm2 + Rr*cp2)*Rinv + eta_2*(up - um)*(up - um);
    const T d     = dsqrt(d2);
    const T uu    = (um + Rr*up)*Rinv;
    const T sm = dmin(uu - d, um - cm);
    const T sp = dmax(uu + d, up + cp);

    // Batten star speed (GPUonly.cuh:857-866)
    const T facm = rm * (sm - um);
    const T facp = rp * (sp - up);
    const T ss = (pp - pm + um*facm - up*facp) / (facm - facp);

    const int s = sign_star_of(ss);
    const T s_minus = dmin((T)0.0f, sm);
    const T s_pluss = dmax((T)0.0f, sp);
    // every flux of this face divides by the same two denominators with the
    // same normal velocities, so chi* is shared (identical operations)
    const T chi_m = (sm - um) / (sm - ss);
    const T chi_p = (sp - up) / (sp - ss);

    // rho, G, P (passive): _hllc_rho (GPUonly.cuh:869-903)
    {
        const T qdm = rm*chi_m - rm, qdp = rp*chi_p - rp;
        o.f[0] = hllc_blend<Pol, true>(s, rm*um + s_minus*qdm, rp*up + s_pluss*qdp);
    }
    {
        const T qdm = Gm*chi_m - Gm, qdp = Gp*chi_p - Gp;
        o.f[5] = hllc_blend<Pol, true>(s, Gm*um + s_minus*qdm, Gp*up + s_pluss*qdp);
    }
    {
        const T qdm = Pm*chi_m - Pm, qdp = Pp*chi_p - Pp;
        o.f[6] = hllc_blend<Pol, true>(s, Pm*um + s_minus*qdm, Pp*up + s_pluss*qdp);
    }
    // normal momentum: _hllc_pvel (GPUonly.cuh:947-984)
    T fn;
    {
        const T qm = rm*um, qp = rp*up;
        const T qdm = rm*ss*chi_m - qm, qdp = rp*ss*chi_p - qp;
        fn = hllc_blend<Pol, false>(s, (qm*um + pm) + s_minus*qdm, (qp*up + pp) + s_pluss*qdp);
    }
    // transverse momenta: _hllc_vel (GPUonly.cuh:906-944)
    T ft1, ft2;
    {
        const T qm = rm*S.t1m, qp = rp*S.t1p;
        const T qdm = qm*chi_m - qm, qdp = qp*chi_p - qp;
        ft1 = hllc_blend<Pol, false>(s, qm*um + s_minus*qdm, qp*up + s_pluss*qdp);
    }
    {
        const T qm = rm*S.t2m, qp = rp*S.t2p;
        const T qdm = qm*chi_m - qm, qdp = qp*chi_p - qp;
        ft2 = hllc_blend<Pol, false>(s, qm*um + s_minus*qdm, qp*up + s_pluss*qdp);
    }
    // energy: _hllc_e (GPUonly.cuh:987-1026)
    {
        const T qm = Gm*pm + Pm + (T)0.5f*rm*(um*um + S.t1m*S.t1m + S.t2m*S.t2m);
        const T qp = Gp*pp + Pp + (T)0.5f*rp*(up*up + S.t1p*S.t1p + S.t2p*S.t2p);
        const T qdm = chi_m*(qm + (ss - um)*(rm*ss + pm/(sm - um))) - qm;
        const T qdp = chi_p*(qp + (ss - up)*(rp*ss + pp/(sp - up))) - qp;
        o.f[4] = hllc_blend<Pol, false>(s, um*(qm + pm) + s_minus*qdm, up*(qp + pp) + s_pluss*qdp);
    }
    // extra-term velocity: _extraterm_hllc_vel (GPUonly.cuh:1029-1042)
    o.vel = hllc_blend<Pol, false>(s, um + s_minus*(chi_m - (T)1.0f), up + s_pluss*(chi_p - (T)1.0f));

    // normal / transverse momenta back to (rho u, rho v, rho w):
    // x: (n, t1, t2), y: (t1, n, t2), z: (t1, t2, n)
    o.f[1] = dir == 0 ? fn : ft1;
    o.f[2] = dir == 1 ? fn : (dir == 0 ? ft1 : ft2);
    o.f[3] = dir == 2 ? fn : ft2;
    o.Gm = Gm; o.Gp = Gp; o.Pm = Pm; o.Pp = Pp;
}

// The same face in the fast policies: every left/right-symmetric quantity is
// one packed pair (lane x = minus / left, lane y = plus / right) and the
// divisions are single-precision reciprocals.  The wave speeds follow
// hllc_face above term by term; the fluxes are the same expressions
// factored: the advected quantities share V = S (chi - 1) + u, and the
// energy flux cancels the (s - u) of chi against the p/(s - u) of the
// reference's star-state energy.
template <class T>
__device__ __forceinline__ void hllc_face_packed(const FaceState<T>& S, const int dir, FaceOut<T>& o)
{
    typedef typename PairOf<T>::V V;
    const V Rh = f2(S.rm, S.rp), Uh = f2(S.nm, S.np), Ph = f2(S.pm, S.pp);
    const V Gh = f2(S.Gm, S.Gp), Qh = f2(S.Pm, S.Pp);
    const V T1 = f2(S.t1m, S.t1p), T2 = f2(S.t2m, S.t2p);
    const T um = S.nm, up = S.np;

    // Einfeldt bounds
    const V ir = rcp2(Rh);
    const T Rr   = dsqrt(S.rp * ir.x);
    const T Rinv = rcp_approx((T)1 + Rr);
    const V c2 = mul2(fma2(add2(Ph, Qh), rcp2(Gh), Ph), ir);
    const T cm = dsqrt(c2.x), cp = dsqrt(c2.y);
    const T eta_2 = (T)0.5 * Rr * Rinv * Rinv;
    const T du = up - um;
    const T d  = dsqrt((c2.x + Rr * c2.y) * Rinv + eta_2 * du * du);
    const T uu = (um + Rr * up) * Rinv;
    const T sm = dmin(uu - d, um - cm);
    const T sp = dmax(uu + d, up + cp);

    // Batten star speed
    const V SU  = sub2(f2(sm, sp), Uh);                       // (sm - um, sp - up)
    const V fac = mul2(Rh, SU);
    const T ss = (S.pp - S.pm + um * fac.x - up * fac.y) * rcp_approx(fac.x - fac.y);
    const int s = sign_star_of(ss);
    const V Sg  = f2(dmin((T)0, sm), dmax((T)0, sp));
    const V SS  = f2s(ss);
    const V Dinv = rcp2(sub2(f2(sm, sp), SS));                // 1/(s - s*)
    const V D   = sub2(SS, Uh);                               // s* - u
    const V C1  = mul2(D, Dinv);                              // chi - 1 = (s* - u)/(s - s*)
    const V Wb  = f2((T)0.5 * (T)(1 + s), (T)0.5 * (T)(1 - s));

    // every advected quantity X has the star-state flux S (X chi - X) + X u
    // = X V with V = S (chi - 1) + u, the extra-term velocity's argument too
    const V A = mul2(Sg, C1);
    const V V_ = add2(A, Uh);
    // rho, G, P (passive)
    o.f[0] = blend2(Wb, mul2(Rh, V_));
    o.f[5] = blend2(Wb, mul2(Gh, V_));
    o.f[6] = blend2(Wb, mul2(Qh, V_));
    // normal momentum: S (rho s* chi - rho u) + rho u^2 + p
    // = rho (S (s* chi - u) + u^2) + p
    const V U2 = mul2(Uh, Uh);
    // (s* chi - u = s* (chi - 1) + s* - u)
    const T fn = blend2(Wb, fma2(Rh, fma2(Sg, fma2(SS, C1, D), U2), Ph));
    // transverse momenta
    const V RV = mul2(Rh, V_);
    const T ft1 = blend2(Wb, mul2(T1, RV));
    const T ft2 = blend2(Wb, mul2(T2, RV));
    // energy: S (chi (Q + (s* - u)(rho s* + p/(s - u))) - Q) + u (Q + p)
    // = Q V + S (s* - u)(rho s* (s - u) + p)/(s - s*) + u p, Q = E
    {
        const V ke = fma2(T2, T2, fma2(T1, T1, U2));
        const V Q  = fma2(mul2(f2s((T)0.5), Rh), ke, fma2(Gh, Ph, Qh));
        const V inner = fma2(mul2(Rh, SS), SU, Ph);
        o.f[4] = blend2(Wb, fma2(Q, V_, fma2(A, inner, mul2(Uh, Ph))));
    }
    // extra-term velocity
    o.vel = blend2(Wb, V_);

    o.f[1] = dir == 0 ? fn : ft1;
    o.f[2] = dir == 1 ? fn : (dir == 0 ? ft1 : ft2);
    o.f[3] = dir == 2 ? fn : ft2;
    o.Gm = S.Gm; o.Gp = S.Gp; o.Pm = S.Pm; o.Pp = S.Pp;
}

// Both edge values of one cell with the reference's WENO3 reconstruction
// (the -D_WENO3_ build, GPUonly.cuh:124-137 for the plus side, 163-176 for
// the minus side), from the cells y1, y2, y3 = l-1, l, l+1:
//   R, the minus side of face l+1/2 (_weno_minus with b, c, d = y1, y2, y3):
//     is0 = (c-b)^2, is1 = (d-c)^2, alpha0 = 1./(3.(is0+eps)^2),
//     alpha1 = 2./(3.(is1+eps)^2), w0 = alpha0/(alpha0+alpha1), w1 = 1.-w0,
//     R = w0 (1.5c - .5b) + w1 (.5c + .5d);
//   L, the plus side of face l-1/2 (_weno_pluss with c, d, e = y1, y2, y3):
//     is0 = (d-e)^2, is1 = (d-c)^2, alpha0 = (1./3.)/(is0+eps)^2,
//     alpha1 = (2./3.)/(is1+eps)^2, w0 = alpha0/(alpha0+alpha1), w1 = 1.-w0,
//     L = w0 (1.5d - .5e) + w1 (.5d + .5c);
// both clipped to [min, max] of y1, y2, y3.  The double literals promote the
// weights' arithmetic and the final combination to double, as in the
// reference.  The squared differences are shared: (y2-y3)^2 is (y3-y2)^2
// bit for bit (rounding to nearest is symmetric under negation).
template <class Pol>
__device__ __forceinline__ void weno3_cell_ref(const typename Pol::T y1, const typename Pol::T y2,
        const typename Pol::T y3, typename Pol::T& R, typename Pol::T& L)
{
    typedef typename Pol::T T;
    const T dl = y2 - y1, dr = y3 - y2;
    const T sl = dl*dl, sr = dr*dr;
    const double el = sl + MPCF_WENOEPS, er = sr + MPCF_WENOEPS;
    const T am0 = (T)(1./(3.*el*el)), am1 = (T)(2./(3.*er*er));
    const T wm0 = am0/(am0 + am1);
    const T wm1 = (T)(1. - wm0);
    const T rm = (T)(wm0*(1.5*y2 - .5*y1) + wm1*(.5*y2 + .5*y3));
    const T ap0 = (T)((1./3.)/(er*er)), ap1 = (T)((2./3.)/(el*el));
    const T wp0 = ap0/(ap0 + ap1);
    const T wp1 = (T)(1. - wp0);
    const T rp = (T)(wp0*(1.5*y2 - .5*y3) + wp1*(.5*y2 + .5*y1));
    const T lo = dmin(dmin(y1, y2), y3);
    const T hi = dmax(dmax(y1, y2), y3);
    R = dmin(dmax(rm, lo), hi);
    L = dmin(dmax(rp, lo), hi);
}

// Both edge values of one cell in the policy's arithmetic.
template <class Pol>
__device__ __forceinline__ void weno_cell(const typename Pol::T y0, const typename Pol::T y1,
        const typename Pol::T y2, const typename Pol::T y3, const typename Pol::T y4,
        typename Pol::T& R, typename Pol::T& L)
{
    if constexpr (Pol::kWeno3)         weno3_cell_ref<Pol>(y1, y2, y3, R, L);
    else if constexpr (Pol::kFastWeno) weno_cell_packed<typename Pol::T>(y0, y1, y2, y3, y4, R, L);
    else                               weno_cell_ref<Pol>(y0, y1, y2, y3, y4, R, L);
}

// Wave speeds and fluxes of one face in the policy's arithmetic.
template <class Pol>
__device__ __forceinline__ void face_hllc(const FaceState<typename Pol::T>& S, const int dir, FaceOut<typename Pol::T>& o)
{
    if constexpr (Pol::kFastWeno) hllc_face_packed<typename Pol::T>(S, dir, o);
    else                          hllc_face<Pol>(S, dir, o);
}

// Conserved (rho, rho u, rho v, rho w, E, G, P) -> primitives (rho, u, v, w,
// p, G, P).  Reference form (GPUkernels.cu:209-244):
//   u = (rho u)/rho, ...;  p = (E - 0.5f*rho*(u*u + v*v + w*w) - P) / G
// in the reference-rounding and FP64 policies.  The fast policies multiply
// by reciprocals.  In the liquid E and P are ~50x the internal energy G p,
// so E - ke - P cancels catastrophically in FP32; the mixed policy recovers
// the pressure in compensated FP32 (comp_pressure below).
// Compensated FP32 pressure recovery p = ((E - P) - ke) / G.  E - P is
// formed as the unevaluated sum s + e of the two-sum algorithm (Knuth; s the
// rounded difference, e its exact rounding error), so the cancellation of E
// against P loses nothing; ke (small against E) is subtracted from s and e
// added back; the quotient is a product with the approximate reciprocal of
// G, corrected once by its residual (num - G q) / G.  Every operation is an
// explicit round-to-nearest instruction, so the result does not depend on
// the translation unit's contraction flags.
__device__ __forceinline__ float comp_pressure(const float E, const float P, const float G, const float ke)
{
    const float s = __fsub_rn(E, P);
    const float z = __fsub_rn(s, E);
    const float e = __fadd_rn(__fsub_rn(E, __fsub_rn(s, z)), __fsub_rn(-P, z));
    const float num = __fadd_rn(__fsub_rn(s, ke), e);
    const float iG = rcp_approx(G);
    const float q = __fmul_rn(num, iG);
    return __fmaf_rn(__fmaf_rn(-G, q, num), iG, q);
}

template <class Pol>
__device__ __forceinline__ void to_primitive(const typename Pol::T c[7], typename Pol::T q[7])
{
    typedef typename Pol::T T;
    q[0] = c[0];
    if constexpr (Pol::kFastWeno)
    {
        const T ir = rcp_approx(c[0]);
        q[1] = c[1] * ir;
        q[2] = c[2] * ir;
        q[3] = c[3] * ir;
        if constexpr (Pol::kCompP)
            q[4] = comp_pressure(c[4], c[6], c[5],
                                 __fmul_rn(__fmaf_rn(c[3], q[3], __fmaf_rn(c[2], q[2], __fmul_rn(c[1], q[1]))), 0.5f));
        else
            q[4] = (c[4] - (T)0.5*c[0]*(q[1]*q[1] + q[2]*q[2] + q[3]*q[3]) - c[6]) * rcp_approx(c[5]);
    }
    else
    {
        q[1] = c[1] / c[0];
        q[2] = c[2] / c[0];
        q[3] = c[3] / c[0];
        q[4] = (c[4] - (T)0.5f*c[0]*(q[1]*q[1] + q[2]*q[2] + q[3]*q[3]) - c[6]) / c[5];
    }
    q[5] = c[5];
    q[6] = c[6];
}

// Maximum of non-negative values through the order of their bit patterns
// (a NaN's pattern orders above every finite value, so it surfaces).
__device__ __forceinline__ void atomic_max_bits(void* p, float v)
{
    atomicMax((unsigned*)p, __float_as_uint(v));
}
__device__ __forceinline__ void atomic_max_bits(void* p, double v)
{
    atomicMax((unsigned long long*)p, (unsigned long long)__double_as_longlong(v));
}
__device__ __forceinline__ float  shfl_max(float v)  { for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o)); return v; }
__device__ __forceinline__ double shfl_max(double v) { for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o)); return v; }

// Maximum characteristic speed of one cell, |u|max + c with
//   p = (E - (ru^2+rv^2+rw^2)*(0.5/rho) - P)/G,  c = sqrt(((p+P)/G + p)/rho)
// (GPUkernels.cu:1182-1222; the mixed policy recovers p in compensated FP32).  Every
// operation is an explicit instruction -- round-to-nearest intrinsics, and
// in the fast policies the approximate reciprocal and square root -- so the
// result is the same whatever the translation unit's contraction and
// division flags: the stand-alone reduction and the one fused into the stage
// kernel agree bit for bit.
template <class Pol>
__device__ __forceinline__ typename Pol::T cell_sos_rn(const typename Pol::T r, const typename Pol::T u,
        const typename Pol::T v, const typename Pol::T w, const typename Pol::T e,
        const typename Pol::T G, const typename Pol::T P)
{
    typedef typename Pol::T T;
    if constexpr (sizeof(T) == 8)
    {
        const double sq = __dadd_rn(__dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v)), __dmul_rn(w, w));
        const double p = __ddiv_rn(__dsub_rn(__dsub_rn(e, __dmul_rn(sq, __ddiv_rn(0.5, r))), P), G);
        const double c = __dsqrt_rn(__ddiv_rn(__dadd_rn(__ddiv_rn(__dadd_rn(p, P), G), p), r));
        return __dadd_rn(c, __ddiv_rn(fmax(fmax(fabs(u), fabs(v)), fabs(w)), r));
    }
    else if constexpr (Pol::kFastWeno)
    {
        // the fast policies: reciprocals and square root of the special-
        // function unit, the compensated pressure in the mixed policy,
        // every operation an explicit instruction (so the two reductions
        // still agree bit for bit)
        const float ir = rcp_approx(r), iG = rcp_approx(G);
        const float sq = __fmaf_rn(w, w, __fmaf_rn(v, v, __fmul_rn(u, u)));
        const float ke = __fmul_rn(sq, __fmul_rn(0.5f, ir));
        float p;
        if constexpr (Pol::kCompP)
            p = comp_pressure(e, P, G, ke);
        else
            p = __fmul_rn(__fsub_rn(__fsub_rn(e, ke), P), iG);
        const float c = sqrt_approx(__fmul_rn(__fmaf_rn(__fadd_rn(p, P), iG, p), ir));
        return __fmaf_rn(fmaxf(fmaxf(fabsf(u), fabsf(v)), fabsf(w)), ir, c);
    }
    else
    {
        // the reference-rounding policy: IEEE division and square root
        static_assert(!Pol::kCompP, "compensated pressure: fast policies only");
        const float sq = __fadd_rn(__fadd_rn(__fmul_rn(u, u), __fmul_rn(v, v)), __fmul_rn(w, w));
        const float p = __fdiv_rn(__fsub_rn(__fsub_rn(e, __fmul_rn(sq, __fdiv_rn(0.5f, r))), P), G);
        const float c = __fsqrt_rn(__fdiv_rn(__fadd_rn(__fdiv_rn(__fadd_rn(p, P), G), p), r));
        return __fadd_rn(c, __fdiv_rn(fmaxf(fmaxf(fabsf(u), fabsf(v)), fabsf(w)), r));
    }
}

} // namespace mpcf
