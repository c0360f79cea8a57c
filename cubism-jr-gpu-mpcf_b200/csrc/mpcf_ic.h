// mpcf_ic.h -- the bubble-cloud initial condition of one cell, shared by the
// device kernel and the host generator so both produce the same state (up
// to the last bit of tanh/sqrt, which the two math libraries may round
// differently).
#pragma once

#include <math.h>
#include "mpcf_types.h"

#ifdef __CUDACC__
#define MPCF_HD __host__ __device__
#else
#define MPCF_HD
#endif

namespace mpcf {

MPCF_HD inline unsigned long long mix64(unsigned long long z)
{
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

// counter-based uniform in [-1, 1) keyed on (seed, cell, component)
MPCF_HD inline double noise_uniform(unsigned long long seed, unsigned long long cell, int comp)
{
    const unsigned long long h = mix64(seed * 0x9e3779b97f4a7c15ULL + cell * 3ULL + (unsigned long long)comp + 0x632be59bd9b4e019ULL);
    return (double)(h >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
}

// Conserved state (rho, rho u, rho v, rho w, E, G, P) of cell (ix,iy,iz),
// linear index `lin`, of a domain with spacing h:
//   phi   = min_k (|x - c_k| - R_k),  x = ((ix,iy,iz) + 0.5) h
//   alpha = 0.5 (1 - tanh(phi / (width h)))   (0 beyond phi > 40 width h)
//   rho, G, P, p: alpha-weighted mixtures of gas and liquid
//   u, v, w: noise * U(-1,1) from the counter hash
//   E = G p + P + rho |u|^2 / 2
MPCF_HD inline void ic_cell(const IcParams& P, const double* bub, int nb, double h,
                            int ix, int iy, int iz, unsigned long long lin, double out[7])
{
    const double Gl = 1.0 / (P.gamma_l - 1.0), Pl = P.gamma_l * P.pc_l / (P.gamma_l - 1.0);
    const double Gg = 1.0 / (P.gamma_g - 1.0), Pg = P.gamma_g * P.pc_g / (P.gamma_g - 1.0);
    const double wid = P.width * h;
    const double x = (ix + 0.5) * h, y = (iy + 0.5) * h, z = (iz + 0.5) * h;
    double phi = 1e300;
    for (int k = 0; k < nb; ++k)
    {
        const double dx = x - bub[4 * k], dy = y - bub[4 * k + 1], dz = z - bub[4 * k + 2];
        const double dd = sqrt(dx * dx + dy * dy + dz * dz) - bub[4 * k + 3];
        phi = dd < phi ? dd : phi;
    }
    const double alpha = (phi > 40.0 * wid) ? 0.0 : 0.5 * (1.0 - tanh(phi / wid));
    const double rho = alpha * P.rho_g + (1.0 - alpha) * P.rho_l;
    const double G   = alpha * Gg + (1.0 - alpha) * Gl;
    const double Pc  = alpha * Pg + (1.0 - alpha) * Pl;
    const double p   = alpha * P.p_g + (1.0 - alpha) * P.p_l;
    const double u = P.noise * noise_uniform(P.seed, lin, 0);
    const double v = P.noise * noise_uniform(P.seed, lin, 1);
    const double w = P.noise * noise_uniform(P.seed, lin, 2);
    out[0] = rho;
    out[1] = rho * u;
    out[2] = rho * v;
    out[3] = rho * w;
    out[4] = G * p + Pc + 0.5 * rho * (u * u + v * v + w * w);
    out[5] = G;
    out[6] = Pc;
}

} // namespace mpcf
