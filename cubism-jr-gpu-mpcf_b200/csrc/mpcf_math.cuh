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
//   PolFast32  float everywhere; WENO weights from single-precision
//              reciprocals, fused multiply-adds allowed.
//   PolMixed   PolFast32 plus the stiffened-gas pressure recovery in FP64
//              and FP64 conservation sums.
//   PolFP64    double storage and arithmetic (the all-FP64 GPU oracle run).
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

struct PolRef32  { typedef float  T; static constexpr bool kFastWeno = false; static constexpr bool kP64 = false; static constexpr bool kRefRounding = true;  static constexpr int id = 0; };
struct PolFast32 { typedef float  T; static constexpr bool kFastWeno = true;  static constexpr bool kP64 = false; static constexpr bool kRefRounding = false; static constexpr int id = 1; };
struct PolMixed  { typedef float  T; static constexpr bool kFastWeno = true;  static constexpr bool kP64 = true;  static constexpr bool kRefRounding = false; static constexpr int id = 2; };
struct PolFP64   { typedef double T; static constexpr bool kFastWeno = false; static constexpr bool kP64 = false; static constexpr bool kRefRounding = true;  static constexpr int id = 3; };

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
__device__ __forceinline__ double rcp_approx(double x) { return 1.0 / x; }

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

// Nonlinear weights (omega0, omega1, omega2) from the three indicators and
// the linear weights (c0, c1, c2) = (1, 6, 3) of the reference.
template <class Pol>
__device__ __forceinline__ void weno_weights(const typename Pol::T is0, const typename Pol::T is1,
                                             const typename Pol::T is2,
                                             typename Pol::T& w0, typename Pol::T& w1, typename Pol::T& w2)
{
    typedef typename Pol::T T;
    const T is0plus = is0 + (T)MPCF_WENOEPS;
    const T is1plus = is1 + (T)MPCF_WENOEPS;
    const T is2plus = is2 + (T)MPCF_WENOEPS;
    T alpha0, alpha1, alpha2;
    if (Pol::kFastWeno)
    {
        // single-precision approximate reciprocal (MUFU); the common factor
        // 1/10 cancels in the normalisation and is dropped
        alpha0 = (T)1 * rcp_approx(is0plus*is0plus);
        alpha1 = (T)6 * rcp_approx(is1plus*is1plus);
        alpha2 = (T)3 * rcp_approx(is2plus*is2plus);
    }
    else
    {
        // the 10.0 literal promotes these to double (GPUonly.cuh:111-113)
        alpha0 = (T)((T)(1)*(((T)1)/(10.0*is0plus*is0plus)));
        alpha1 = (T)((T)(6)*(((T)1)/(10.0*is1plus*is1plus)));
        alpha2 = (T)((T)(3)*(((T)1)/(10.0*is2plus*is2plus)));
    }
    const T alphasum = alpha0 + alpha1 + alpha2;
    T inv;
    if (Pol::kFastWeno) inv = rcp_approx(alphasum);
    else                inv = ((T)1)/alphasum;
    w0 = alpha0 * inv;
    w1 = alpha1 * inv;
    w2 = 1 - w0 - w1;
}

// Minus-side (left state) reconstruction at face i-1/2 from cells
// a..e = i-3..i+1, clipped to [min,max] of b,c,d (GPUonly.cuh:138-194).
template <class Pol>
__device__ __forceinline__ typename Pol::T weno_minus_clipped(const typename Pol::T a, const typename Pol::T b,
        const typename Pol::T c, const typename Pol::T d, const typename Pol::T e)
{
    typedef typename Pol::T T;
    const T is0 = beta_f<T>(a, b, c);
    const T is1 = beta_h<T>(b, c, d);
    const T is2 = beta_g<T>(c, d, e);
    T w0, w1, w2;
    weno_weights<Pol>(is0, is1, is2, w0, w1, w2);
    const T r = w0*((T)(1.0/3.)*a-(T)(7./6.)*b+(T)(11./6.)*c) + w1*(-(T)(1./6.)*b+(T)(5./6.)*c+(T)(1./3.)*d) + w2*((T)(1./3.)*c+(T)(5./6.)*d-(T)(1./6.)*e);
    const T mn = dmin(dmin(b, c), d);
    const T mx = dmax(dmax(b, c), d);
    return dmin(dmax(r, mn), mx);
}

// Plus-side (right state) reconstruction at face i-1/2 from cells
// b..f = i-2..i+2, clipped to [min,max] of c,d,e (GPUonly.cuh:99-135,177-183).
template <class Pol>
__device__ __forceinline__ typename Pol::T weno_pluss_clipped(const typename Pol::T b, const typename Pol::T c,
        const typename Pol::T d, const typename Pol::T e, const typename Pol::T f)
{
    typedef typename Pol::T T;
    const T is0 = beta_g<T>(d, e, f);
    const T is1 = beta_h<T>(c, d, e);
    const T is2 = beta_f<T>(b, c, d);
    T w0, w1, w2;
    weno_weights<Pol>(is0, is1, is2, w0, w1, w2);
    const T r = w0*((T)(1./3.)*f-(T)(7./6.)*e+(T)(11./6.)*d) + w1*(-(T)(1./6.)*e+(T)(5./6.)*d+(T)(1./3.)*c) + w2*((T)(1./3.)*d+(T)(5./6.)*c-(T)(1./6.)*b);
    const T mn = dmin(dmin(c, d), e);
    const T mx = dmax(dmax(c, d), e);
    return dmin(dmax(r, mn), mx);
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

// Wave speeds + HLLC fluxes for direction DIR (GPUkernels.cu:255-289 for x,
// :636-668 for y, :932-963 for z; GPUonly.cuh:802-1042).
template <class Pol, int DIR>
__device__ __forceinline__ void hllc_face(const FaceState<typename Pol::T>& S, FaceOut<typename Pol::T>& o)
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

    // scatter normal / transverse momenta to (rho u, rho v, rho w)
    if (DIR == 0)      { o.f[1] = fn;  o.f[2] = ft1; o.f[3] = ft2; }
    else if (DIR == 1) { o.f[1] = ft1; o.f[2] = fn;  o.f[3] = ft2; }
    else               { o.f[1] = ft1; o.f[2] = ft2; o.f[3] = fn;  }
    o.Gm = Gm; o.Gp = Gp; o.Pm = Pm; o.Pp = Pp;
}

// Full face: fetch(q, j) returns primitive q of stencil cell j (j = 0..5 for
// cells i-3..i+2 around face i-1/2).
template <class Pol, int DIR, class Fetch>
__device__ __forceinline__ void face_flux(const Fetch& fetch, FaceOut<typename Pol::T>& o)
{
    typedef typename Pol::T T;
    FaceState<T> S;
    // component indices of the normal / transverse velocities (1=u,2=v,3=w)
    constexpr int qn  = 1 + DIR;
    constexpr int qt1 = DIR == 0 ? 2 : 1;
    constexpr int qt2 = DIR == 2 ? 2 : 3;
#define MPCF_RECON(q, M, P) { \
        const T s0 = fetch(q, 0), s1 = fetch(q, 1), s2 = fetch(q, 2), \
                s3 = fetch(q, 3), s4 = fetch(q, 4), s5 = fetch(q, 5); \
        M = weno_minus_clipped<Pol>(s0, s1, s2, s3, s4); \
        P = weno_pluss_clipped<Pol>(s1, s2, s3, s4, s5); }
    MPCF_RECON(0,   S.rm,  S.rp);
    MPCF_RECON(qn,  S.nm,  S.np);
    MPCF_RECON(qt1, S.t1m, S.t1p);
    MPCF_RECON(qt2, S.t2m, S.t2p);
    MPCF_RECON(4,   S.pm,  S.pp);
    MPCF_RECON(5,   S.Gm,  S.Gp);
    MPCF_RECON(6,   S.Pm,  S.Pp);
#undef MPCF_RECON
    hllc_face<Pol, DIR>(S, o);
}

// Conserved (rho, rho u, rho v, rho w, E, G, P) -> primitives (rho, u, v, w,
// p, G, P).  Reference form (GPUkernels.cu:209-244):
//   u = (rho u)/rho, ...;  p = (E - 0.5f*rho*(u*u + v*v + w*w) - P) / G
// The mixed policy evaluates the pressure recovery in FP64 from the stored
// conserved values: p = (E - 0.5*((rho u)^2+(rho v)^2+(rho w)^2)/rho - P)/G.
template <class Pol>
__device__ __forceinline__ void to_primitive(const typename Pol::T c[7], typename Pol::T q[7])
{
    typedef typename Pol::T T;
    q[0] = c[0];
    q[1] = c[1] / c[0];
    q[2] = c[2] / c[0];
    q[3] = c[3] / c[0];
    if (Pol::kP64)
    {
        const double r = (double)c[0];
        const double ke = 0.5 * ((double)c[1]*(double)c[1] + (double)c[2]*(double)c[2] + (double)c[3]*(double)c[3]) / r;
        q[4] = (T)(((double)c[4] - ke - (double)c[6]) / (double)c[5]);
    }
    else
    {
        q[4] = (c[4] - (T)0.5f*c[0]*(q[1]*q[1] + q[2]*q[2] + q[3]*q[3]) - c[6]) / c[5];
    }
    q[5] = c[5];
    q[6] = c[6];
}

} // namespace mpcf
