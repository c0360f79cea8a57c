/*
 * oracle_ic.h -- CPU restatement of the reference's shock-induced
 * cloud-collapse initial condition.  TEST INFRASTRUCTURE (the checker of the
 * GPU generator, never the product).  Included by oracle.c once per REAL
 * (float: the reference's _FLOAT_PRECISION_ build; double: its double build).
 *
 * Follows, in the reference's evaluation order and types (REAL = the
 * reference's Real; double where the reference's literals promote):
 *   post-shock state (Johnsen)      source/Sim/Sim_SICCloudMPI.cpp:85-103
 *   shock normal normalisation      Sim_SICCloudMPI.cpp:76-81
 *   is_shock, heaviside              Sim_SICCloudMPI.cpp:204-217, Types.h:90-93
 *   set_IC (mixture, energy)         Sim_SICCloudMPI.cpp:247-276
 *   shape distance, cloud indicator  Sim_SICCloudMPI.h:97-101, 285-301
 *   get_IC, Simpson 3x3x3 average    Sim_SICCloudMPI.cpp:279-337
 *   cell loop (_ic_quad)             Sim_SICCloudMPI.cpp:339-357
 * prm[] order: rho0 u0 p0 rhoB uB pB pressure_ratio nx ny nz Sx Sy Sz g1 g2 pc1 pc2.
 */

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

typedef struct
{
    REAL rho0, u0, p0, rhoB, uB, pB, psi;
    REAL n[3], S[3];
    REAL g1, g2, pc1, pc2;
    REAL rho1, u1, p1, mach;
} SFX(sic_state);

static void SFX(sic_setup)(const double* prm, SFX(sic_state)* st)
{
    st->rho0 = (REAL)prm[0]; st->u0 = (REAL)prm[1]; st->p0 = (REAL)prm[2];
    st->rhoB = (REAL)prm[3]; st->uB = (REAL)prm[4]; st->pB = (REAL)prm[5];
    st->psi  = (REAL)prm[6];
    for (int i = 0; i < 3; ++i) { st->n[i] = (REAL)prm[7 + i]; st->S[i] = (REAL)prm[10 + i]; }
    st->g1 = (REAL)prm[13]; st->g2 = (REAL)prm[14]; st->pc1 = (REAL)prm[15]; st->pc2 = (REAL)prm[16];
    /* |n| with pow(Real, int) promoted to double */
    const REAL mag = (REAL)sqrt((double)st->n[0] * (double)st->n[0] + (double)st->n[1] * (double)st->n[1]
                                + (double)st->n[2] * (double)st->n[2]);
    for (int i = 0; i < 3; ++i) st->n[i] /= mag;

    const REAL gamma = st->g1, pc = st->pc1, p0 = st->p0, rho0 = st->rho0, u0 = st->u0, psi = st->psi;
    const REAL p1   = p0 * psi;
    const REAL tmp1 = (REAL)(((double)gamma + 1.0) / ((double)gamma - 1.0));
    const REAL tmp2 = (p1 + pc) / (p0 + pc);
    const REAL c0   = RSQRT(gamma * (p0 + pc) / rho0);
    const REAL mach = (REAL)sqrt(((double)gamma + 1.0) / (2.0 * (double)gamma) * ((double)psi - 1.0) * (double)p0
                                 / (double)(p0 + pc) + 1.0);
    st->mach = mach;
    st->u1   = (REAL)((double)u0 + (double)c0 * ((double)psi - 1.0) * (double)p0 / (double)(gamma * (p0 + pc) * mach));
    st->rho1 = (REAL)((double)rho0 * ((double)(tmp1 * tmp2) + 1.0) / (double)(tmp1 + tmp2));
    st->p1   = p1;
}

/* sphere distance |pos - c| - r: differences in Real, squares and sum in
 * double (pow(Real, 2) promotes), result stored as Real */
static REAL SFX(sic_shape_eval)(const REAL* shp, const REAL pos[3])
{
    const double dx = (double)(pos[0] - shp[0]), dy = (double)(pos[1] - shp[1]), dz = (double)(pos[2] - shp[2]);
    return (REAL)(sqrt(dx * dx + dy * dy + dz * dz) - (double)shp[3]);
}

/* cloud indicator: cosine ramp of half-width eps around the nearest surface
 * (eps = 0: 1 inside or on a sphere, 0 outside) */
static REAL SFX(sic_eval)(const REAL* shapes, int nshapes, const REAL pos[3], double eps)
{
    REAL d = (REAL)HUGE_VAL;
    for (int i = 0; i < nshapes; ++i)
    {
        const REAL nd = SFX(sic_shape_eval)(shapes + 4 * i, pos);
        d = (nd < d) ? nd : d;                                   /* std::min(d, nd) */
    }
    const double x = (double)((double)d + eps) / (2 * eps);
    const double mx = (0. < x) ? x : 0.;                         /* std::max(0., x) */
    const double mn = (mx < 1.) ? mx : 1.;                       /* std::min(1., .) */
    const double alpha = M_PI * mn;
    return (REAL)(0.5 + 0.5 * cos(alpha));
}

static void SFX(sic_set_ic)(const SFX(sic_state)* st, const REAL shock, const REAL bubble, REAL out[7])
{
    const REAL G1 = st->g1 - 1, G2 = st->g2 - 1;
    const REAL F1 = st->g1 * st->pc1, F2 = st->g2 * st->pc2;
    const REAL rho = shock * st->rho1 + (1 - shock) * (st->rhoB * bubble + st->rho0 * (1 - bubble));
    const REAL u   = (shock * st->u1 + (1 - shock) * (st->uB * bubble + st->u0 * (1 - bubble))) * rho;
    const REAL v = 0, w = 0;
    const REAL G = (REAL)(1. / (double)G1 * (double)(1 - bubble) + 1. / (double)G2 * (double)bubble);
    const REAL P = F1 / G1 * (1 - bubble) + F2 / G2 * bubble;
    const REAL pressure = shock * st->p1 + (1 - shock) * (st->pB * bubble + st->p0 * (1 - bubble));
    const REAL ke = (REAL)(0.5 * (double)(u * u + v * v + w * w) / (double)rho);
    out[0] = rho; out[1] = u; out[2] = v; out[3] = w;
    out[4] = pressure * G + P + ke;
    out[5] = G; out[6] = P;
}

static void SFX(sic_get_ic)(const SFX(sic_state)* st, const REAL* shapes, int nshapes, double eps,
                            const REAL pos[3], REAL out[7])
{
    const REAL d = -(st->n[0] * (st->S[0] - pos[0]) + st->n[1] * (st->S[1] - pos[1]) + st->n[2] * (st->S[2] - pos[2]));
    const REAL shock = d > 0 ? (REAL)0 : (REAL)1;
    const REAL bubble = nshapes > 0 ? SFX(sic_eval)(shapes, nshapes, pos, eps) : (REAL)0;
    SFX(sic_set_ic)(st, shock, bubble, out);
}

/* 3x3x3 Simpson average over the cell of centre p, samples h apart
 * (h = half the grid spacing), z then y then x; weights stored as Real */
static void SFX(sic_integral)(const SFX(sic_state)* st, const REAL* shapes, int nshapes, double eps,
                              const double p[3], const REAL h, REAL out[7])
{
    const REAL w6 = (REAL)(1 / 6.), w23 = (REAL)(2. / 3);
    REAL smp[3][3][3][7], zi[3][3][7], yi[3][7];
    const REAL x0[3] = {(REAL)(p[0] - (double)h), (REAL)(p[1] - (double)h), (REAL)(p[2] - (double)h)};
    for (int iz = 0; iz < 3; ++iz)
        for (int iy = 0; iy < 3; ++iy)
            for (int ix = 0; ix < 3; ++ix)
            {
                const REAL pos[3] = {x0[0] + (REAL)ix * h, x0[1] + (REAL)iy * h, x0[2] + (REAL)iz * h};
                SFX(sic_get_ic)(st, shapes, nshapes, eps, pos, smp[iz][iy][ix]);
            }
    for (int iy = 0; iy < 3; ++iy)
        for (int ix = 0; ix < 3; ++ix)
            for (int m = 0; m < 7; ++m)
                zi[iy][ix][m] = (w6 * smp[0][iy][ix][m] + w23 * smp[1][iy][ix][m]) + w6 * smp[2][iy][ix][m];
    for (int ix = 0; ix < 3; ++ix)
        for (int m = 0; m < 7; ++m)
            yi[ix][m] = (w6 * zi[0][ix][m] + w23 * zi[1][ix][m]) + w6 * zi[2][ix][m];
    for (int m = 0; m < 7; ++m)
        out[m] = (w6 * yi[0][m] + w23 * yi[1][m]) + w6 * yi[2][m];
}
