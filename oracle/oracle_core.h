/*
 * oracle_core.h -- CPU restatement of the reference's per-stage hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: it is compiled
 * into oracle/liboracle.so and called from tests/, from
 * __graft_entry__.smoke() and from bench.py's CPU-baseline leg.  The product
 * (the CUDA library under cubism-jr-gpu-mpcf_b200/) never includes, links or
 * calls it.
 *
 * Included twice by oracle.c with
 *     REAL  = float  | double
 *     SFX(name)      appends _f32 | _f64
 *     RMIN/RMAX/RSQRT/RABS = the libm functions of that width
 *
 * Every function follows the reference source operation for operation in C
 * evaluation order (left-to-right, usual arithmetic conversions), so the
 * double-promoted sub-expressions of the FP32 reference are reproduced
 * exactly.  The file must be compiled with -ffp-contract=off and without
 * -ffast-math: the oracle's rounding is the literal C semantics of the
 * reference source with no multiply-add contraction.
 *
 * Reference files (paths inside the reference project):
 *   source/GPU/GPUonly.cuh       WENO5, clipping, Einfeldt, HLLC, extra term
 *   source/GPU/GPUkernels.cu     flux pipelines, extra terms, divergence,
 *                                update, max speed of sound
 *   source/BoundaryConditions.h  absorbing / reflecting ghost fills
 *   source/GPUlab.cpp            single-chunk process_all data flow
 *   source/LSRK3_IntegratorMPI.cpp  LSRK3 coefficients and dt
 */

/* ---------------------------------------------------------------------- */
/* WENO5-JS reconstruction: GPUonly.cuh:99-135 (plus), :138-174 (minus)    */
/* ---------------------------------------------------------------------- */
static REAL SFX(weno_pluss)(const REAL b, const REAL c, const REAL d, const REAL e, const REAL f)
{
    if (g_oracle_weno3)
    {
        /* the reference's _WENO3_ build (GPUonly.cuh:125-137): the WENOEPS
         * and fraction literals promote the weights and the result to double */
        const REAL is0 = (d-e)*(d-e);
        const REAL is1 = (d-c)*(d-c);
        const REAL alpha0 = (1./3.)/((is0+ORACLE_WENOEPS)*(is0+ORACLE_WENOEPS));
        const REAL alpha1 = (2./3.)/((is1+ORACLE_WENOEPS)*(is1+ORACLE_WENOEPS));
        const REAL omega0 = alpha0/(alpha0+alpha1);
        const REAL omega1 = 1.-omega0;
        return omega0*(1.5*d-.5*e) + omega1*(.5*d+.5*c);
    }
    const REAL is0 = d*(d*(REAL)(10./3.)- e*(REAL)(31./3.) + f*(REAL)(11./3.)) + e*(e*(REAL)(25./3.) - f*(REAL)(19./3.)) +    f*f*(REAL)(4./3.);
    const REAL is1 = c*(c*(REAL)(4./3.) - d*(REAL)(13./3.) + e*(REAL)(5./3.)) + d*(d*(REAL)(13./3.)  - e*(REAL)(13./3.)) +    e*e*(REAL)(4./3.);
    const REAL is2 = b*(b*(REAL)(4./3.) - c*(REAL)(19./3.) + d*(REAL)(11./3.)) + c*(c*(REAL)(25./3.) - d*(REAL)(31./3.)) +    d*d*(REAL)(10./3.);

    const REAL is0plus = is0 + (REAL)ORACLE_WENOEPS;
    const REAL is1plus = is1 + (REAL)ORACLE_WENOEPS;
    const REAL is2plus = is2 + (REAL)ORACLE_WENOEPS;

    /* the 10.0 literal promotes these three to double (GPUonly.cuh:111-113) */
    const REAL alpha0 = (REAL)(1)*(((REAL)1)/(10.0*is0plus*is0plus));
    const REAL alpha1 = (REAL)(6)*(((REAL)1)/(10.0*is1plus*is1plus));
    const REAL alpha2 = (REAL)(3)*(((REAL)1)/(10.0*is2plus*is2plus));
    const REAL alphasum = alpha0+alpha1+alpha2;

    const REAL omega0=alpha0 * (((REAL)1)/alphasum);
    const REAL omega1=alpha1 * (((REAL)1)/alphasum);
    const REAL omega2= 1-omega0-omega1;

    return omega0*((REAL)(1./3.)*f-(REAL)(7./6.)*e+(REAL)(11./6.)*d) + omega1*(-(REAL)(1./6.)*e+(REAL)(5./6.)*d+(REAL)(1./3.)*c) + omega2*((REAL)(1./3.)*d+(REAL)(5./6.)*c-(REAL)(1./6.)*b);
}

static REAL SFX(weno_minus)(const REAL a, const REAL b, const REAL c, const REAL d, const REAL e)
{
    if (g_oracle_weno3)
    {
        /* _WENO3_ (GPUonly.cuh:164-176); note 1./(3.*x*x) here against
         * (1./3.)/(x*x) on the plus side */
        const REAL is0 = (c-b)*(c-b);
        const REAL is1 = (d-c)*(d-c);
        const REAL alpha0 = 1./(3.*(is0+ORACLE_WENOEPS)*(is0+ORACLE_WENOEPS));
        const REAL alpha1 = 2./(3.*(is1+ORACLE_WENOEPS)*(is1+ORACLE_WENOEPS));
        const REAL omega0=alpha0/(alpha0+alpha1);
        const REAL omega1=1.-omega0;
        return omega0*(1.5*c-.5*b) + omega1*(.5*c+.5*d);
    }
    const REAL is0 = a*(a*(REAL)(4./3.)  - b*(REAL)(19./3.)  + c*(REAL)(11./3.)) + b*(b*(REAL)(25./3.)  - c*(REAL)(31./3.)) + c*c*(REAL)(10./3.);
    const REAL is1 = b*(b*(REAL)(4./3.)  - c*(REAL)(13./3.)  + d*(REAL)(5./3.))  + c*(c*(REAL)(13./3.)  - d*(REAL)(13./3.)) + d*d*(REAL)(4./3.);
    const REAL is2 = c*(c*(REAL)(10./3.) - d*(REAL)(31./3.)  + e*(REAL)(11./3.)) + d*(d*(REAL)(25./3.)  - e*(REAL)(19./3.)) + e*e*(REAL)(4./3.);

    const REAL is0plus = is0 + (REAL)ORACLE_WENOEPS;
    const REAL is1plus = is1 + (REAL)ORACLE_WENOEPS;
    const REAL is2plus = is2 + (REAL)ORACLE_WENOEPS;

    /* double-promoted, GPUonly.cuh:150-152 */
    const REAL alpha0 = (REAL)(1)*(((REAL)1)/(10.0*is0plus*is0plus));
    const REAL alpha1 = (REAL)(6)*(((REAL)1)/(10.0*is1plus*is1plus));
    const REAL alpha2 = (REAL)(3)*(((REAL)1)/(10.0*is2plus*is2plus));
    const REAL alphasum = alpha0+alpha1+alpha2;

    const REAL omega0=alpha0 * (((REAL)1)/alphasum);
    const REAL omega1=alpha1 * (((REAL)1)/alphasum);
    const REAL omega2= 1-omega0-omega1;

    return omega0*((REAL)(1.0/3.)*a-(REAL)(7./6.)*b+(REAL)(11./6.)*c) + omega1*(-(REAL)(1./6.)*b+(REAL)(5./6.)*c+(REAL)(1./3.)*d) + omega2*((REAL)(1./3.)*c+(REAL)(5./6.)*d-(REAL)(1./6.)*e);
}

/* GPUonly.cuh:177-194 */
static REAL SFX(weno_pluss_clipped)(const REAL b, const REAL c, const REAL d, const REAL e, const REAL f)
{
    const REAL retval = SFX(weno_pluss)(b,c,d,e,f);
    const REAL min_in = RMIN( RMIN(c,d), e );
    const REAL max_in = RMAX( RMAX(c,d), e );
    return RMIN(RMAX(retval, min_in), max_in);
}

static REAL SFX(weno_minus_clipped)(const REAL a, const REAL b, const REAL c, const REAL d, const REAL e)
{
    const REAL retval = SFX(weno_minus)(a,b,c,d,e);
    const REAL min_in = RMIN( RMIN(b,c), d );
    const REAL max_in = RMAX( RMAX(b,c), d );
    return RMIN(RMAX(retval, min_in), max_in);
}

/* ---------------------------------------------------------------------- */
/* Wave speeds and HLLC fluxes: GPUonly.cuh:802-1042                       */
/* ---------------------------------------------------------------------- */
static void SFX(char_vel_einfeldt)(const REAL rm, const REAL rp,
        const REAL vm, const REAL vp, const REAL pm, const REAL pp,
        const REAL Gm, const REAL Gp, const REAL Pm, const REAL Pp,
        REAL* outm, REAL* outp)
{
    const REAL Rr   = RSQRT(rp / rm);
    const REAL Rinv = 1.0f / (1.0f + Rr);
    const REAL cm2 = ((pm + Pm)/Gm + pm) / rm;
    const REAL cp2 = ((pp + Pp)/Gp + pp) / rp;
    const REAL cm  = RSQRT(cm2);
    const REAL cp  = RSQRT(cp2);
    const REAL um    = vm;
    const REAL up    = vp;
    const REAL eta_2 = 0.5f*Rr*Rinv*Rinv;
    const REAL d2    = (cm2 + Rr*cp2)*Rinv + eta_2*(up - um)*(up - um);
    const REAL d     = RSQRT(d2);
    const REAL u     = (um + Rr*up)*Rinv;
    *outm = RMIN(u - d, um - cm);
    *outp = RMAX(u + d, up + cp);
}

static REAL SFX(char_vel_star)(const REAL rm, const REAL rp,
        const REAL vm, const REAL vp, const REAL pm, const REAL pp,
        const REAL sm, const REAL sp)
{
    const REAL facm = rm * (sm - vm);
    const REAL facp = rp * (sp - vp);
    return (pp - pm + vm*facm - vp*facp) / (facm - facp);
}

static int SFX(sign_of)(const REAL ss) { return ss == 0 ? 0 : (ss < 0 ? -1 : 1); }

/* GPUonly.cuh:869-903; note the double literal 0.5 in the second weight */
static REAL SFX(hllc_rho)(const REAL rm, const REAL rp, const REAL vm, const REAL vp,
        const REAL sm, const REAL sp, const REAL ss)
{
    const int sign_star = SFX(sign_of)(ss);
    const REAL s_minus = RMIN(0.0f, sm);
    const REAL s_pluss = RMAX(0.0f, sp);
    const REAL chi_starm = (sm - vm) / (sm - ss);
    const REAL chi_starp = (sp - vp) / (sp - ss);
    const REAL qm        = rm;
    const REAL qp        = rp;
    const REAL q_deltam  = qm*chi_starm - qm;
    const REAL q_deltap  = qp*chi_starp - qp;
    const REAL fm = qm*vm;
    const REAL fp = qp*vp;
    const REAL flux = (0.5f*(1 + sign_star)) * (fm + s_minus*q_deltam) + (0.5*(1 - sign_star)) * (fp + s_pluss*q_deltap);
    return flux;
}

/* GPUonly.cuh:906-944 */
static REAL SFX(hllc_vel)(const REAL rm,  const REAL rp, const REAL vm,  const REAL vp,
        const REAL vdm, const REAL vdp, const REAL sm,  const REAL sp,  const REAL ss)
{
    const int sign_star = SFX(sign_of)(ss);
    const REAL s_minus  = RMIN(0.0f, sm);
    const REAL s_pluss  = RMAX(0.0f, sp);
    const REAL chi_starm = (sm - vdm) / (sm - ss);
    const REAL chi_starp = (sp - vdp) / (sp - ss);
    const REAL qm        = rm*vm;
    const REAL qp        = rp*vp;
    const REAL q_deltam  = qm*chi_starm - qm;
    const REAL q_deltap  = qp*chi_starp - qp;
    const REAL fm = qm*vdm;
    const REAL fp = qp*vdp;
    const REAL flux = (0.5f*(1 + sign_star)) * (fm + s_minus*q_deltam) + (0.5f*(1 - sign_star)) * (fp + s_pluss*q_deltap);
    return flux;
}

/* GPUonly.cuh:947-984 */
static REAL SFX(hllc_pvel)(const REAL rm, const REAL rp, const REAL vm, const REAL vp,
        const REAL pm, const REAL pp, const REAL sm, const REAL sp, const REAL ss)
{
    const int sign_star = SFX(sign_of)(ss);
    const REAL s_minus  = RMIN(0.0f, sm);
    const REAL s_pluss  = RMAX(0.0f, sp);
    const REAL chi_starm = (sm - vm) / (sm - ss);
    const REAL chi_starp = (sp - vp) / (sp - ss);
    const REAL qm        = rm*vm;
    const REAL qp        = rp*vp;
    const REAL q_deltam  = rm*ss*chi_starm - qm;
    const REAL q_deltap  = rp*ss*chi_starp - qp;
    const REAL fm = qm*vm + pm;
    const REAL fp = qp*vp + pp;
    const REAL flux = (0.5f*(1 + sign_star)) * (fm + s_minus*q_deltam) + (0.5f*(1 - sign_star)) * (fp + s_pluss*q_deltap);
    return flux;
}

/* GPUonly.cuh:987-1026 */
static REAL SFX(hllc_e)(const REAL rm,  const REAL rp, const REAL vdm, const REAL vdp,
        const REAL v1m, const REAL v1p, const REAL v2m, const REAL v2p,
        const REAL pm,  const REAL pp, const REAL Gm,  const REAL Gp,
        const REAL Pm,  const REAL Pp, const REAL sm,  const REAL sp,  const REAL ss)
{
    const int sign_star = SFX(sign_of)(ss);
    const REAL s_minus  = RMIN(0.0f, sm);
    const REAL s_pluss  = RMAX(0.0f, sp);
    const REAL chi_starm = (sm - vdm) / (sm - ss);
    const REAL chi_starp = (sp - vdp) / (sp - ss);
    const REAL qm        = Gm*pm + Pm + 0.5f*rm*(vdm*vdm + v1m*v1m + v2m*v2m);
    const REAL qp        = Gp*pp + Pp + 0.5f*rp*(vdp*vdp + v1p*v1p + v2p*v2p);
    const REAL q_deltam  = chi_starm*(qm + (ss - vdm)*(rm*ss + pm/(sm - vdm))) - qm;
    const REAL q_deltap  = chi_starp*(qp + (ss - vdp)*(rp*ss + pp/(sp - vdp))) - qp;
    const REAL fm = vdm*(qm + pm);
    const REAL fp = vdp*(qp + pp);
    const REAL flux = (0.5f*(1 + sign_star)) * (fm + s_minus*q_deltam) + (0.5f*(1 - sign_star)) * (fp + s_pluss*q_deltap);
    return flux;
}

/* GPUonly.cuh:1029-1042 */
static REAL SFX(extraterm_hllc_vel)(const REAL um, const REAL up,
        const REAL Gm, const REAL Gp, const REAL Pm, const REAL Pp,
        const REAL sm, const REAL sp, const REAL ss)
{
    const int sign_star   = (ss == 0) ? 0 : ((ss < 0) ? -1 : 1);
    const REAL s_minus   = RMIN(0.0f, sm);
    const REAL s_pluss   = RMAX(0.0f, sp);
    const REAL chi_starm = (sm - um)/(sm - ss) - 1.0f;
    const REAL chi_starp = (sp - up)/(sp - ss) - 1.0f;
    (void)Gm; (void)Gp; (void)Pm; (void)Pp;
    return (0.5f*(1 + sign_star))*(um + s_minus*chi_starm) + (0.5f*(1 - sign_star))*(up + s_pluss*chi_starp);
}

/* ---------------------------------------------------------------------- */
/* One face: stencil -> primitives -> WENO -> wave speeds -> HLLC          */
/* GPUkernels.cu:184-290 (x), :565-669 (y), :874-964 (z).                  */
/* s[q][j], q = 0..6 (rho, rho u, rho v, rho w, E, G, P), j = 0..5 the     */
/* cells i-3 .. i+2 around face i-1/2.  dir 0/1/2 = x/y/z.                 */
/* out[0..6] = fluxes (r,u,v,w,e,G,P), out[7..11] = Gm,Gp,Pm,Pp,u*.        */
/* ---------------------------------------------------------------------- */
static void SFX(face_flux)(REAL s[7][6], const int dir, REAL out[12])
{
    REAL* r = s[0];
    REAL* u = s[1];
    REAL* v = s[2];
    REAL* w = s[3];
    REAL* e = s[4];
    REAL* G = s[5];
    REAL* P = s[6];
    REAL p[6];
    int j;

    const REAL rp = SFX(weno_pluss_clipped)(r[1], r[2], r[3], r[4], r[5]);
    const REAL rm = SFX(weno_minus_clipped)(r[0], r[1], r[2], r[3], r[4]);
    for (j = 0; j < 6; ++j) u[j] /= r[j];
    const REAL up = SFX(weno_pluss_clipped)(u[1], u[2], u[3], u[4], u[5]);
    const REAL um = SFX(weno_minus_clipped)(u[0], u[1], u[2], u[3], u[4]);
    for (j = 0; j < 6; ++j) v[j] /= r[j];
    const REAL vp = SFX(weno_pluss_clipped)(v[1], v[2], v[3], v[4], v[5]);
    const REAL vm = SFX(weno_minus_clipped)(v[0], v[1], v[2], v[3], v[4]);
    for (j = 0; j < 6; ++j) w[j] /= r[j];
    const REAL wp = SFX(weno_pluss_clipped)(w[1], w[2], w[3], w[4], w[5]);
    const REAL wm = SFX(weno_minus_clipped)(w[0], w[1], w[2], w[3], w[4]);
    for (j = 0; j < 6; ++j)
        p[j] = (e[j] - 0.5f*r[j]*(u[j]*u[j] + v[j]*v[j] + w[j]*w[j]) - P[j]) / G[j];
    const REAL pp = SFX(weno_pluss_clipped)(p[1], p[2], p[3], p[4], p[5]);
    const REAL pm = SFX(weno_minus_clipped)(p[0], p[1], p[2], p[3], p[4]);
    const REAL Gp = SFX(weno_pluss_clipped)(G[1], G[2], G[3], G[4], G[5]);
    const REAL Gm = SFX(weno_minus_clipped)(G[0], G[1], G[2], G[3], G[4]);
    const REAL Pp = SFX(weno_pluss_clipped)(P[1], P[2], P[3], P[4], P[5]);
    const REAL Pm = SFX(weno_minus_clipped)(P[0], P[1], P[2], P[3], P[4]);

    REAL sm, sp, ss;
    REAL fr, fu, fv, fw, fe, fG, fP, vel;
    if (dir == 0)
    {
        SFX(char_vel_einfeldt)(rm, rp, um, up, pm, pp, Gm, Gp, Pm, Pp, &sm, &sp);
        ss = SFX(char_vel_star)(rm, rp, um, up, pm, pp, sm, sp);
        fr = SFX(hllc_rho)(rm, rp, um, up, sm, sp, ss);
        fu = SFX(hllc_pvel)(rm, rp, um, up, pm, pp, sm, sp, ss);
        fv = SFX(hllc_vel)(rm, rp, vm, vp, um, up, sm, sp, ss);
        fw = SFX(hllc_vel)(rm, rp, wm, wp, um, up, sm, sp, ss);
        fe = SFX(hllc_e)(rm, rp, um, up, vm, vp, wm, wp, pm, pp, Gm, Gp, Pm, Pp, sm, sp, ss);
        fG = SFX(hllc_rho)(Gm, Gp, um, up, sm, sp, ss);
        fP = SFX(hllc_rho)(Pm, Pp, um, up, sm, sp, ss);
        vel = SFX(extraterm_hllc_vel)(um, up, Gm, Gp, Pm, Pp, sm, sp, ss);
    }
    else if (dir == 1)
    {
        SFX(char_vel_einfeldt)(rm, rp, vm, vp, pm, pp, Gm, Gp, Pm, Pp, &sm, &sp);
        ss = SFX(char_vel_star)(rm, rp, vm, vp, pm, pp, sm, sp);
        fr = SFX(hllc_rho)(rm, rp, vm, vp, sm, sp, ss);
        fu = SFX(hllc_vel)(rm, rp, um, up, vm, vp, sm, sp, ss);
        fv = SFX(hllc_pvel)(rm, rp, vm, vp, pm, pp, sm, sp, ss);
        fw = SFX(hllc_vel)(rm, rp, wm, wp, vm, vp, sm, sp, ss);
        fe = SFX(hllc_e)(rm, rp, vm, vp, um, up, wm, wp, pm, pp, Gm, Gp, Pm, Pp, sm, sp, ss);
        fG = SFX(hllc_rho)(Gm, Gp, vm, vp, sm, sp, ss);
        fP = SFX(hllc_rho)(Pm, Pp, vm, vp, sm, sp, ss);
        vel = SFX(extraterm_hllc_vel)(vm, vp, Gm, Gp, Pm, Pp, sm, sp, ss);
    }
    else
    {
        SFX(char_vel_einfeldt)(rm, rp, wm, wp, pm, pp, Gm, Gp, Pm, Pp, &sm, &sp);
        ss = SFX(char_vel_star)(rm, rp, wm, wp, pm, pp, sm, sp);
        fr = SFX(hllc_rho)(rm, rp, wm, wp, sm, sp, ss);
        fu = SFX(hllc_vel)(rm, rp, um, up, wm, wp, sm, sp, ss);
        fv = SFX(hllc_vel)(rm, rp, vm, vp, wm, wp, sm, sp, ss);
        fw = SFX(hllc_pvel)(rm, rp, wm, wp, pm, pp, sm, sp, ss);
        fe = SFX(hllc_e)(rm, rp, wm, wp, um, up, vm, vp, pm, pp, Gm, Gp, Pm, Pp, sm, sp, ss);
        fG = SFX(hllc_rho)(Gm, Gp, wm, wp, sm, sp, ss);
        fP = SFX(hllc_rho)(Pm, Pp, wm, wp, sm, sp, ss);
        vel = SFX(extraterm_hllc_vel)(wm, wp, Gm, Gp, Pm, Pp, sm, sp, ss);
    }
    out[0] = fr; out[1] = fu; out[2] = fv; out[3] = fw;
    out[4] = fe; out[5] = fG; out[6] = fP;
    out[7] = Gm; out[8] = Gp; out[9] = Pm; out[10] = Pp; out[11] = vel;
}

/* ---------------------------------------------------------------------- */
/* Ghost fills: BoundaryConditions.h:60-109.                               */
/* gx[side][q][GHOSTMAPX(ix,iy,iz)]  ix 0..2 (3*NY*NZ)                     */
/* gy[side][q][GHOSTMAPY(ix,iy,iz)]  iy 0..2 (NX*3*NZ)                     */
/* gz[side][q][ID3(ix,iy,iz,NX,NY)]  iz 0..2 (NX*NY*3)                     */
/* side 0 = left: layer 0 is the outermost cell (-3);                      */
/* side 1 = right: layer 0 is the innermost ghost (N).                     */
/* ---------------------------------------------------------------------- */
static void SFX(fill_ghosts)(const int NX, const int NY, const int NZ, const int bc[6],
        REAL* const* U, REAL* gx[2][7], REAL* gy[2][7], REAL* gz[2][7])
{
    int side, q, ix, iy, iz;
    for (side = 0; side < 2; ++side)
    for (q = 0; q < 7; ++q)
    {
        /* x faces */
        {
            const int refl = bc[0 + side] == 1;
            const REAL fac = (refl && q == 1) ? (REAL)-1 : (REAL)1;
            for (iz = 0; iz < NZ; ++iz)
            for (iy = 0; iy < NY; ++iy)
            for (ix = 0; ix < 3; ++ix)
            {
                int sx;
                if (refl) sx = side == 0 ? 2 - ix : NX - 1 - ix;
                else      sx = side == 0 ? 0 : NX - 1;
                const REAL val = U[q][sx + NX * (iy + NY * iz)];
                gx[side][q][ix + 3 * (iy + NY * iz)] = refl ? fac * val : val;
            }
        }
        /* y faces */
        {
            const int refl = bc[2 + side] == 1;
            const REAL fac = (refl && q == 2) ? (REAL)-1 : (REAL)1;
            for (iz = 0; iz < NZ; ++iz)
            for (iy = 0; iy < 3; ++iy)
            for (ix = 0; ix < NX; ++ix)
            {
                int sy;
                if (refl) sy = side == 0 ? 2 - iy : NY - 1 - iy;
                else      sy = side == 0 ? 0 : NY - 1;
                const REAL val = U[q][ix + NX * (sy + NY * iz)];
                gy[side][q][ix + NX * (iy + 3 * iz)] = refl ? fac * val : val;
            }
        }
        /* z faces */
        {
            const int refl = bc[4 + side] == 1;
            const REAL fac = (refl && q == 3) ? (REAL)-1 : (REAL)1;
            for (iz = 0; iz < 3; ++iz)
            for (iy = 0; iy < NY; ++iy)
            for (ix = 0; ix < NX; ++ix)
            {
                int sz;
                if (refl) sz = side == 0 ? 2 - iz : NZ - 1 - iz;
                else      sz = side == 0 ? 0 : NZ - 1;
                const REAL val = U[q][ix + NX * (iy + NY * sz)];
                gz[side][q][ix + NX * (iy + NY * iz)] = refl ? fac * val : val;
            }
        }
    }
}

/* cell value with ghosts: x/y from the compact ghost buffers
 * (GPUonly.cuh:305-510), z from the ghost slices (GPUlab.cpp:742-761) */
static REAL SFX(cell)(const int NX, const int NY, const int NZ, REAL* const* U,
        REAL* gx[2][7], REAL* gy[2][7], REAL* gz[2][7],
        const int q, const int ix, const int iy, const int iz)
{
    if (ix < 0)   return gx[0][q][(ix + 3) + 3 * (iy + NY * iz)];
    if (ix >= NX) return gx[1][q][(ix - NX) + 3 * (iy + NY * iz)];
    if (iy < 0)   return gy[0][q][ix + NX * ((iy + 3) + 3 * iz)];
    if (iy >= NY) return gy[1][q][ix + NX * ((iy - NY) + 3 * iz)];
    if (iz < 0)   return gz[0][q][ix + NX * (iy + NY * (iz + 3))];
    if (iz >= NZ) return gz[1][q][ix + NX * (iy + NY * (iz - NZ))];
    return U[q][ix + NX * (iy + NY * iz)];
}

/* ---------------------------------------------------------------------- */
/* One LSRK3 stage over the whole block, single chunk:                     */
/* GPUlab::process_all (GPUlab.cpp:703-793) with nslices == NZ, i.e.       */
/* _xflux/_xextraterm, _yflux/_yextraterm, _zflux/_zextraterm,             */
/* _divergence, _update (GPUkernels.cu:35-1179).                           */
/* On return U holds U + b*rhs and R holds rhs = a*R - dtinvh*L(U).        */
/* ---------------------------------------------------------------------- */
static int SFX(stage)(const int NX, const int NY, const int NZ, const int bc[6],
        REAL* const* U, REAL* const* R, const REAL a, const REAL b, const REAL dtinvh)
{
    const size_t N = (size_t)NX * NY * NZ;
    const size_t NFX = (size_t)(NX + 1) * NY * NZ;
    const size_t NFY = (size_t)NX * (NY + 1) * NZ;
    const size_t NFZ = (size_t)NX * NY * (NZ + 1);
    REAL* gx[2][7]; REAL* gy[2][7]; REAL* gz[2][7];
    REAL* fx[12]; REAL* fy[12]; REAL* fz[12];
    REAL *sumG, *sumP, *divU;
    REAL* rhs[7];
    int q, ok = 1;

    for (q = 0; q < 7; ++q)
    {
        gx[0][q] = (REAL*)malloc(sizeof(REAL) * 3 * NY * NZ);
        gx[1][q] = (REAL*)malloc(sizeof(REAL) * 3 * NY * NZ);
        gy[0][q] = (REAL*)malloc(sizeof(REAL) * NX * 3 * NZ);
        gy[1][q] = (REAL*)malloc(sizeof(REAL) * NX * 3 * NZ);
        gz[0][q] = (REAL*)malloc(sizeof(REAL) * NX * NY * 3);
        gz[1][q] = (REAL*)malloc(sizeof(REAL) * NX * NY * 3);
        rhs[q]   = (REAL*)malloc(sizeof(REAL) * N);
        ok = ok && gx[0][q] && gx[1][q] && gy[0][q] && gy[1][q] && gz[0][q] && gz[1][q] && rhs[q];
    }
    for (q = 0; q < 12; ++q)
    {
        fx[q] = (REAL*)malloc(sizeof(REAL) * NFX);
        fy[q] = (REAL*)malloc(sizeof(REAL) * NFY);
        fz[q] = (REAL*)malloc(sizeof(REAL) * NFZ);
        ok = ok && fx[q] && fy[q] && fz[q];
    }
    sumG = (REAL*)malloc(sizeof(REAL) * N);
    sumP = (REAL*)malloc(sizeof(REAL) * N);
    divU = (REAL*)malloc(sizeof(REAL) * N);
    ok = ok && sumG && sumP && divU;

    if (ok)
    {
        SFX(fill_ghosts)(NX, NY, NZ, bc, U, gx, gy, gz);

        /* face fluxes in x, y, z (GPUkernels.cu:104-290, 483-669, 847-964) */
        /* (iz, iy) rows shared out together: balanced for thin slabs too */
        #pragma omp parallel for collapse(2) schedule(static)
        for (int iz = 0; iz < NZ + 1; ++iz)
        for (int iy = 0; iy < NY + 1; ++iy)
        {
            REAL s[7][6];
            REAL out[12];
            for (int ix = 0; ix < NX + 1; ++ix)
            {
                int dir;
                for (dir = 0; dir < 3; ++dir)
                {
                    const int ex = dir == 0 ? NX + 1 : NX;
                    const int ey = dir == 1 ? NY + 1 : NY;
                    const int ez = dir == 2 ? NZ + 1 : NZ;
                    if (ix >= ex || iy >= ey || iz >= ez) continue;
                    for (int qq = 0; qq < 7; ++qq)
                    for (int j = 0; j < 6; ++j)
                    {
                        const int o = j - 3;
                        s[qq][j] = SFX(cell)(NX, NY, NZ, U, gx, gy, gz, qq,
                                ix + (dir == 0 ? o : 0), iy + (dir == 1 ? o : 0), iz + (dir == 2 ? o : 0));
                    }
                    SFX(face_flux)(s, dir, out);
                    const size_t idx = (size_t)ix + (size_t)ex * (iy + (size_t)ey * iz);
                    REAL** f = dir == 0 ? fx : (dir == 1 ? fy : fz);
                    for (int k = 0; k < 12; ++k) f[k][idx] = out[k];
                }
            }
        }

        /* extra terms (GPUkernels.cu:35-62 "=", :422-444 and :795-817 "+="),
         * divergence (:1092-1139) and update (:1142-1179) */
        #pragma omp parallel for collapse(2) schedule(static)
        for (int iz = 0; iz < NZ; ++iz)
        for (int iy = 0; iy < NY; ++iy)
        for (int ix = 0; ix < NX; ++ix)
        {
            const size_t idx  = (size_t)ix + (size_t)NX * (iy + (size_t)NY * iz);
            const size_t ixm = (size_t)ix + (size_t)(NX + 1) * (iy + (size_t)NY * iz);
            const size_t ixp = ixm + 1;
            const size_t iym = (size_t)ix + (size_t)NX * (iy + (size_t)(NY + 1) * iz);
            const size_t iyp = iym + NX;
            const size_t izm = idx;
            const size_t izp = idx + (size_t)NX * NY;
            const REAL factor6 = 1.0f / 6.0f;
            int k;

            sumG[idx] = fx[8][ixm] + fx[7][ixp];
            sumP[idx] = fx[10][ixm] + fx[9][ixp];
            divU[idx] = fx[11][ixp] - fx[11][ixm];
            sumG[idx] += fy[8][iym] + fy[7][iyp];
            sumP[idx] += fy[10][iym] + fy[9][iyp];
            divU[idx] += fy[11][iyp] - fy[11][iym];
            sumG[idx] += fz[8][izm] + fz[7][izp];
            sumP[idx] += fz[10][izm] + fz[9][izp];
            divU[idx] += fz[11][izp] - fz[11][izm];

            for (k = 0; k < 7; ++k)
            {
                const REAL fxp = fx[k][ixp], fxm = fx[k][ixm];
                const REAL fyp = fy[k][iyp], fym = fy[k][iym];
                const REAL fzp = fz[k][izp], fzm = fz[k][izm];
                REAL rhs_k;
                if (k == 5)
                    rhs_k = dtinvh*(fxp - fxm + fyp - fym + fzp - fzm   - divU[idx] * sumG[idx] * factor6);
                else if (k == 6)
                    rhs_k = dtinvh*(fxp - fxm + fyp - fym + fzp - fzm   - divU[idx] * sumP[idx] * factor6);
                else
                    rhs_k = dtinvh*(fxp - fxm + fyp - fym + fzp - fzm);
                rhs[k][idx] = a*R[k][idx] - rhs_k;
            }
        }

        /* _update writes b*rhs + U (into d_tmp, copied to pdata);
         * the rhs is copied into ptmp (GPUlab.cpp:772-788) */
        #pragma omp parallel for schedule(static)
        for (long long i = 0; i < (long long)N; ++i)
        {
            for (int k = 0; k < 7; ++k)
            {
                U[k][i] = b*rhs[k][i] + U[k][i];
                R[k][i] = rhs[k][i];
            }
        }
    }

    for (q = 0; q < 7; ++q)
    {
        free(gx[0][q]); free(gx[1][q]); free(gy[0][q]); free(gy[1][q]);
        free(gz[0][q]); free(gz[1][q]); free(rhs[q]);
    }
    for (q = 0; q < 12; ++q) { free(fx[q]); free(fy[q]); free(fz[q]); }
    free(sumG); free(sumP); free(divU);
    return ok ? 0 : -1;
}

/* ---------------------------------------------------------------------- */
/* Max speed of sound, GPU formula: _maxSOS, GPUkernels.cu:1182-1222       */
/* ---------------------------------------------------------------------- */
static REAL SFX(max_sos)(const long long N, REAL* const* U)
{
    /* per-thread maxima, then their maximum: the maximum of a set does not
     * depend on the order it is taken in */
    REAL sos = 0;
    #pragma omp parallel
    {
    REAL loc = 0;
    long long i;
    #pragma omp for schedule(static)
    for (i = 0; i < N; ++i)
    {
        const REAL r = U[0][i];
        const REAL u = U[1][i];
        const REAL v = U[2][i];
        const REAL w = U[3][i];
        const REAL e = U[4][i];
        const REAL G = U[5][i];
        const REAL P = U[6][i];
        const REAL p = (e - (u*u + v*v + w*w)*(0.5f/r) - P) / G;
        const REAL c = RSQRT(((p + P) / G + p) / r);
        loc = RMAX(loc, c + RMAX(RMAX(RABS(u), RABS(v)), RABS(w)) / r);
    }
    #pragma omp critical
    sos = RMAX(sos, loc);
    }
    return sos;
}

/* Max speed of sound, CPU formula: MaxSpeedOfSound.cpp:18-55 (0.5/r is a
 * double literal there) */
static REAL SFX(max_sos_cpp)(const long long N, REAL* const* U)
{
    REAL sos = 0;
    long long i;
    for (i = 0; i < N; ++i)
    {
        const REAL r = U[0][i];
        const REAL u = U[1][i];
        const REAL v = U[2][i];
        const REAL w = U[3][i];
        const REAL e = U[4][i];
        const REAL G = U[5][i];
        const REAL P = U[6][i];
        const REAL p = (e - (u*u + v*v + w*w)*(0.5/r) - P)/G;
        const REAL c = RSQRT(((p+P)/G+p)/r);
        const REAL cand = c + RMAX(RMAX(RABS(u), RABS(v)), RABS(w))/r;
        sos = sos < cand ? cand : sos;   /* std::max(sos, cand) */
    }
    return sos;
}

/* ---------------------------------------------------------------------- */
/* One LSRK3 step: LSRK3_IntegratorMPI.cpp:27-62 on one rank with the      */
/* CUDA sound-speed kernel.  Returns dt.                                   */
/* ---------------------------------------------------------------------- */
static double SFX(step)(const int NX, const int NY, const int NZ, const int bc[6],
        REAL* const* U, REAL* const* R, const double cfl, const double dt_max, const double h,
        double* sos_out)
{
    /* the FP32 reference keeps sos as a float (LSRK3_IntegratorMPI.h:18);
     * the FP64 variant keeps it in double */
    const REAL sos = SFX(max_sos)((long long)NX * NY * NZ, U);
    double dt = cfl*h/sos;
    dt = dt_max < dt ? dt_max : dt;
    if (sos_out) *sos_out = (double)sos;
    if (SFX(stage)(NX, NY, NZ, bc, U, R, (REAL)0, (REAL)(1./4), (REAL)(dt/h))) return -1.0;
    if (SFX(stage)(NX, NY, NZ, bc, U, R, (REAL)(-17./32), (REAL)(8./9), (REAL)(dt/h))) return -1.0;
    if (SFX(stage)(NX, NY, NZ, bc, U, R, (REAL)(-32./27), (REAL)(3./4), (REAL)(dt/h))) return -1.0;
    return dt;
}
