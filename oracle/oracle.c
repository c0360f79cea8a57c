/*
 * oracle.c -- exported entry points of the CPU parity oracle.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle_core.h).  Built by oracle/Makefile
 * into oracle/liboracle.so with -O2 -ffp-contract=off -fopenmp; loaded by
 * tests/ and bench.py (CPU-baseline leg) through ctypes.  The CUDA product
 * never links it.
 *
 * Layout of every field array: 7 SoA fields (rho, rho*u, rho*v, rho*w, E,
 * G, P), cell (ix,iy,iz) at ix + NX*(iy + NY*iz)  (Types.h:31,
 * NodeBlock.h:26-36).  bc[6] = {x-left, x-right, y-left, y-right, z-left,
 * z-right}, 0 = absorbing, 1 = reflecting (BoundaryConditions.h:60-109).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* WENOEPS: Makefile.config:15,252 (weps ?= 1e-6) */
#define ORACLE_WENOEPS 1e-6

/* reconstruction order: 0 WENO5 (the default build), 1 the reference's
 * compile-time _WENO3_ build (GPUonly.cuh:102,141) */
static int g_oracle_weno3 = 0;
void oracle_set_weno3(int on) { g_oracle_weno3 = on != 0; }

/* ---- single precision ---- */
#define REAL float
#define SFX(name) name##_f32
#define RMIN fminf
#define RMAX fmaxf
#define RSQRT sqrtf
#define RABS fabsf
#include "oracle_core.h"
#include "oracle_ic.h"
#undef REAL
#undef SFX
#undef RMIN
#undef RMAX
#undef RSQRT
#undef RABS

/* ---- double precision (the CPU twin of the all-FP64 GPU path) ---- */
#define REAL double
#define SFX(name) name##_f64
#define RMIN fmin
#define RMAX fmax
#define RSQRT sqrt
#define RABS fabs
#include "oracle_core.h"
#include "oracle_ic.h"
#undef REAL
#undef SFX
#undef RMIN
#undef RMAX
#undef RSQRT
#undef RABS

/* --------------------------------------------------------------------- */
int oracle_stage_f32(int nx, int ny, int nz, const int* bc, float** U, float** R,
                     float a, float b, float dtinvh)
{ return stage_f32(nx, ny, nz, bc, U, R, a, b, dtinvh); }

int oracle_stage_f64(int nx, int ny, int nz, const int* bc, double** U, double** R,
                     double a, double b, double dtinvh)
{ return stage_f64(nx, ny, nz, bc, U, R, a, b, dtinvh); }

float oracle_max_sos_f32(long long n, float** U) { return max_sos_f32(n, U); }
double oracle_max_sos_f64(long long n, double** U) { return max_sos_f64(n, U); }
float oracle_max_sos_cpp_f32(long long n, float** U) { return max_sos_cpp_f32(n, U); }

double oracle_step_f32(int nx, int ny, int nz, const int* bc, float** U, float** R,
                       double cfl, double dt_max, double h, double* sos_out)
{ return step_f32(nx, ny, nz, bc, U, R, cfl, dt_max, h, sos_out); }

double oracle_step_f64(int nx, int ny, int nz, const int* bc, double** U, double** R,
                       double cfl, double dt_max, double h, double* sos_out)
{ return step_f64(nx, ny, nz, bc, U, R, cfl, dt_max, h, sos_out); }

/* Ghost fills alone, for cross-checking against the reference's own
 * BoundaryConditions.h compiled in oracle/_ref.  Buffers are laid out
 * [side][q][...] contiguously: gx 2*7*3*NY*NZ, gy 2*7*NX*3*NZ,
 * gz 2*7*NX*NY*3. */
void oracle_fill_ghosts_f32(int nx, int ny, int nz, const int* bc, float** U,
                            float* gx_all, float* gy_all, float* gz_all)
{
    float* gx[2][7]; float* gy[2][7]; float* gz[2][7];
    const size_t sx = (size_t)3 * ny * nz, sy = (size_t)nx * 3 * nz, sz = (size_t)nx * ny * 3;
    for (int s = 0; s < 2; ++s)
        for (int q = 0; q < 7; ++q)
        {
            gx[s][q] = gx_all + (s * 7 + q) * sx;
            gy[s][q] = gy_all + (s * 7 + q) * sy;
            gz[s][q] = gz_all + (s * 7 + q) * sz;
        }
    fill_ghosts_f32(nx, ny, nz, bc, U, gx, gy, gz);
}

/* One face flux from a raw 7x6 stencil (conserved variables), for unit
 * tests of the face pipeline.  s_flat[q*6 + j]. */
void oracle_face_flux_f32(const float* s_flat, int dir, float* out)
{
    float s[7][6];
    memcpy(s, s_flat, sizeof(s));
    face_flux_f32(s, dir, out);
}

float oracle_weno_minus_clipped_f32(float a, float b, float c, float d, float e)
{ return weno_minus_clipped_f32(a, b, c, d, e); }
float oracle_weno_pluss_clipped_f32(float b, float c, float d, float e, float f)
{ return weno_pluss_clipped_f32(b, c, d, e, f); }

/* Single functions of the face pipeline, exported for pinning against the
 * reference's own GPUonly.cuh compiled on the host (oracle/_ref). */
void oracle_char_vel_einfeldt_f32(float rm, float rp, float vm, float vp, float pm, float pp,
                                  float Gm, float Gp, float Pm, float Pp, float* out2)
{ char_vel_einfeldt_f32(rm, rp, vm, vp, pm, pp, Gm, Gp, Pm, Pp, &out2[0], &out2[1]); }
float oracle_char_vel_star_f32(float rm, float rp, float vm, float vp, float pm, float pp, float sm, float sp)
{ return char_vel_star_f32(rm, rp, vm, vp, pm, pp, sm, sp); }
float oracle_hllc_rho_f32(float rm, float rp, float vm, float vp, float sm, float sp, float ss)
{ return hllc_rho_f32(rm, rp, vm, vp, sm, sp, ss); }
float oracle_hllc_vel_f32(float rm, float rp, float vm, float vp, float vdm, float vdp, float sm, float sp, float ss)
{ return hllc_vel_f32(rm, rp, vm, vp, vdm, vdp, sm, sp, ss); }
float oracle_hllc_pvel_f32(float rm, float rp, float vm, float vp, float pm, float pp, float sm, float sp, float ss)
{ return hllc_pvel_f32(rm, rp, vm, vp, pm, pp, sm, sp, ss); }
float oracle_hllc_e_f32(float rm, float rp, float vdm, float vdp, float v1m, float v1p, float v2m, float v2p,
                        float pm, float pp, float Gm, float Gp, float Pm, float Pp, float sm, float sp, float ss)
{ return hllc_e_f32(rm, rp, vdm, vdp, v1m, v1p, v2m, v2p, pm, pp, Gm, Gp, Pm, Pp, sm, sp, ss); }
float oracle_extraterm_hllc_vel_f32(float um, float up, float Gm, float Gp, float Pm, float Pp, float sm, float sp, float ss)
{ return extraterm_hllc_vel_f32(um, up, Gm, Gp, Pm, Pp, sm, sp, ss); }

/* Stencil of face i-1/2 in direction dir around (ix,iy,iz), from the state
 * plus the ghost buffers of oracle_fill_ghosts_f32's layout. */
void oracle_stencil_f32(int nx, int ny, int nz, float** U, const float* gx_all, const float* gy_all,
                        const float* gz_all, int q, int dir, int ix, int iy, int iz, float* out6)
{
    float* gx[2][7]; float* gy[2][7]; float* gz[2][7];
    const size_t sx = (size_t)3 * ny * nz, sy = (size_t)nx * 3 * nz, sz = (size_t)nx * ny * 3;
    for (int s = 0; s < 2; ++s)
        for (int k = 0; k < 7; ++k)
        {
            gx[s][k] = (float*)gx_all + (s * 7 + k) * sx;
            gy[s][k] = (float*)gy_all + (s * 7 + k) * sy;
            gz[s][k] = (float*)gz_all + (s * 7 + k) * sz;
        }
    for (int j = 0; j < 6; ++j)
    {
        const int o = j - 3;
        out6[j] = cell_f32(nx, ny, nz, U, gx, gy, gz, q, ix + (dir == 0 ? o : 0), iy + (dir == 1 ? o : 0), iz + (dir == 2 ? o : 0));
    }
}

/* --------------------------------------------------------------------- */
/* Shock-induced cloud-collapse IC (oracle_ic.h) on an nx*ny*nz block of
 * spacing 1/max(nx,ny,nz), cell centres (i+0.5)h (NodeBlock.h:71,90-96).
 * shapes4: nshapes x (cx, cy, cz, r), rounded to Real as the reference's
 * cloud.dat reader does.  post4 (optional): rho1, u1, p1, mach. */
#define ORACLE_SIC(SUF, T)                                                               \
void oracle_sic_cloud_##SUF(int nx, int ny, int nz, const double* prm, int nshapes,      \
                            const double* shapes4, double eps, T** out7, double* post4) \
{                                                                                         \
    sic_state_##SUF st;                                                                   \
    sic_setup_##SUF(prm, &st);                                                            \
    if (post4) { post4[0] = st.rho1; post4[1] = st.u1; post4[2] = st.p1; post4[3] = st.mach; } \
    T* shp = (T*)malloc(sizeof(T) * 4 * (nshapes > 0 ? nshapes : 1));                      \
    for (int i = 0; i < 4 * nshapes; ++i) shp[i] = (T)shapes4[i];                          \
    const int mx = nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz);                   \
    const double hd = 1.0 / mx;                                                           \
    const T h = (T)hd;                                                                    \
    _Pragma("omp parallel for")                                                           \
    for (int iz = 0; iz < nz; ++iz)                                                       \
        for (int iy = 0; iy < ny; ++iy)                                                   \
            for (int ix = 0; ix < nx; ++ix)                                               \
            {                                                                             \
                const double p[3] = {hd * (ix + 0.5), hd * (iy + 0.5), hd * (iz + 0.5)};  \
                T v[7];                                                                   \
                sic_integral_##SUF(&st, shp, nshapes, eps, p, h / 2, v);                  \
                const long long c = ix + (long long)nx * (iy + (long long)ny * iz);       \
                for (int m = 0; m < 7; ++m) out7[m][c] = v[m];                            \
            }                                                                             \
    free(shp);                                                                            \
}
ORACLE_SIC(f32, float)
ORACLE_SIC(f64, double)
