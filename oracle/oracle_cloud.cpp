/*
 * oracle_cloud.cpp -- CPU restatement of the benchmark workloads' bubble-cloud
 * set-up: seeded rejection sampling of non-overlapping spheres and the
 * tanh-smoothed liquid / gas initial condition.
 *
 * TEST INFRASTRUCTURE ONLY.  Linked into oracle/liboracle.so; the tests
 * check it against the library's host generator (mpcf_ic_cloud_host,
 * mpcf_bubbles), and bench.py's reference arm uses it to build its CPU
 * sample without loading the product library.  The CUDA product never links
 * it.
 *
 * Placement: std::mt19937_64 seeded with `seed`; every uniform is the top 53
 * bits of one draw, u = a + (b - a) * (draw >> 11) * 2^-53; per attempt x, y,
 * z, then r; a sphere is kept when its distance to every kept sphere is at
 * least r + r_k + gap.
 *
 * Cell (ix, iy, iz) of a domain of spacing h = 1 / max(global extent), centre
 * x = (i + 0.5) h in global coordinates:
 *   phi   = min_k (|x - c_k| - R_k)
 *   alpha = 0.5 (1 - tanh(phi / (width h)))   (0 beyond phi > 40 width h)
 *   rho, G, P, p: alpha-weighted mixtures of the gas and liquid values,
 *   G = 1/(gamma - 1), P = gamma pc / (gamma - 1)
 *   u, v, w = noise * U(-1, 1), a counter hash (splitmix64 finaliser) of
 *   (seed, global linear cell index, component)
 *   E = G p + P + rho |u|^2 / 2
 * Every operation is in double in the order written; the result is rounded
 * to the storage type once.
 */
#include <math.h>
#include <random>

namespace {

unsigned long long mix64(unsigned long long z)
{
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

double noise_uniform(unsigned long long seed, unsigned long long cell, int comp)
{
    const unsigned long long h = mix64(seed * 0x9e3779b97f4a7c15ULL + cell * 3ULL + (unsigned long long)comp
                                       + 0x632be59bd9b4e019ULL);
    return (double)(h >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
}

/* prm: rho_l p_l gamma_l pc_l rho_g p_g gamma_g pc_g noise width */
void cloud_cell(const double* prm, unsigned long long seed, const double* bub, int nb, double h,
                long long ix, long long iy, long long iz, unsigned long long lin, double out[7])
{
    const double rho_l = prm[0], p_l = prm[1], gamma_l = prm[2], pc_l = prm[3];
    const double rho_g = prm[4], p_g = prm[5], gamma_g = prm[6], pc_g = prm[7];
    const double noise = prm[8], width = prm[9];
    const double Gl = 1.0 / (gamma_l - 1.0), Pl = gamma_l * pc_l / (gamma_l - 1.0);
    const double Gg = 1.0 / (gamma_g - 1.0), Pg = gamma_g * pc_g / (gamma_g - 1.0);
    const double wid = width * h;
    const double x = (ix + 0.5) * h, y = (iy + 0.5) * h, z = (iz + 0.5) * h;
    double phi = 1e300;
    for (int k = 0; k < nb; ++k)
    {
        const double dx = x - bub[4 * k], dy = y - bub[4 * k + 1], dz = z - bub[4 * k + 2];
        const double dd = sqrt(dx * dx + dy * dy + dz * dz) - bub[4 * k + 3];
        phi = dd < phi ? dd : phi;
    }
    const double alpha = (phi > 40.0 * wid) ? 0.0 : 0.5 * (1.0 - tanh(phi / wid));
    const double rho = alpha * rho_g + (1.0 - alpha) * rho_l;
    const double G   = alpha * Gg + (1.0 - alpha) * Gl;
    const double Pc  = alpha * Pg + (1.0 - alpha) * Pl;
    const double p   = alpha * p_g + (1.0 - alpha) * p_l;
    const double u = noise * noise_uniform(seed, lin, 0);
    const double v = noise * noise_uniform(seed, lin, 1);
    const double w = noise * noise_uniform(seed, lin, 2);
    out[0] = rho;
    out[1] = rho * u;
    out[2] = rho * v;
    out[3] = rho * w;
    out[4] = G * p + Pc + 0.5 * rho * (u * u + v * v + w * w);
    out[5] = G;
    out[6] = Pc;
}

template <class T>
void cloud_block(int nx, int ny, int nz, const int* org3, const int* glob3, const double* prm,
                 unsigned long long seed, int nb, const double* bub4, T** out7)
{
    const int gx = glob3 ? glob3[0] : nx, gy = glob3 ? glob3[1] : ny, gz = glob3 ? glob3[2] : nz;
    const int ox = org3 ? org3[0] : 0, oy = org3 ? org3[1] : 0, oz = org3 ? org3[2] : 0;
    const int m = gx > gy ? (gx > gz ? gx : gz) : (gy > gz ? gy : gz);
    const double h = 1.0 / (double)m;
#pragma omp parallel for schedule(static)
    for (int iz = 0; iz < nz; ++iz)
        for (int iy = 0; iy < ny; ++iy)
            for (int ix = 0; ix < nx; ++ix)
            {
                const long long X = ox + ix, Y = oy + iy, Z = oz + iz;
                const unsigned long long lin = (unsigned long long)(X + (long long)gx * (Y + (long long)gy * Z));
                double c[7];
                cloud_cell(prm, seed, bub4, nb, h, X, Y, Z, lin, c);
                const long long i = ix + (long long)nx * (iy + (long long)ny * iz);
                for (int q = 0; q < 7; ++q) out7[q][i] = (T)c[q];
            }
}

} // namespace

extern "C" {

/* Seeded non-overlapping spheres (x, y, z, r) into out4; returns how many
 * were placed within max_tries attempts (<= 0: 100000). */
int oracle_bubbles(unsigned long long seed, int n, double rmin, double rmax, const double* lo3,
                   const double* hi3, double gap, int max_tries, double* out4)
{
    std::mt19937_64 rng(seed);
    auto uni = [&](double a, double b) { return a + (b - a) * ((double)(rng() >> 11) * (1.0 / 9007199254740992.0)); };
    int placed = 0;
    const int tries = max_tries > 0 ? max_tries : 100000;
    for (int t = 0; t < tries && placed < n; ++t)
    {
        const double x = uni(lo3[0], hi3[0]), y = uni(lo3[1], hi3[1]), z = uni(lo3[2], hi3[2]);
        const double r = uni(rmin, rmax);
        bool ok = true;
        for (int k = 0; k < placed && ok; ++k)
        {
            const double dx = x - out4[4 * k], dy = y - out4[4 * k + 1], dz = z - out4[4 * k + 2];
            ok = sqrt(dx * dx + dy * dy + dz * dz) >= r + out4[4 * k + 3] + gap;
        }
        if (!ok) continue;
        out4[4 * placed] = x; out4[4 * placed + 1] = y; out4[4 * placed + 2] = z; out4[4 * placed + 3] = r;
        ++placed;
    }
    return placed;
}

/* Cloud state of an nx*ny*nz block whose cell (0,0,0) is global cell org3
 * of a glob3 domain (null: the block is the whole domain). */
void oracle_ic_cloud_f32(int nx, int ny, int nz, const int* org3, const int* glob3, const double* prm,
                         unsigned long long seed, int nb, const double* bub4, float** out7)
{ cloud_block<float>(nx, ny, nz, org3, glob3, prm, seed, nb, bub4, out7); }

void oracle_ic_cloud_f64(int nx, int ny, int nz, const int* org3, const int* glob3, const double* prm,
                         unsigned long long seed, int nb, const double* bub4, double** out7)
{ cloud_block<double>(nx, ny, nz, org3, glob3, prm, seed, nb, bub4, out7); }

}
