/*
 * ref_lsrk3_driver.cpp -- drives the B200 path through the reference's own,
 * unchanged LSRK3 integrator.  TEST INFRASTRUCTURE: built by
 * `make -C oracle ref` into oracle/_ref/libref_lsrk3_driver.so, linking
 *   source/LSRK3_IntegratorMPI.cpp  (the reference's time integrator, as is)
 *   source/MaxSpeedOfSound.cpp      (the reference's CPU sound speed, as is)
 * against the drop-in shim (cubism-jr-gpu-mpcf_b200/shim: GridMPI, GPUlab,
 * BoundaryConditions, single-rank mpi.h) and libmpcf_b200.so.  The shim
 * headers shadow the reference's own GPUlab.h/GridMPI.h/Types.h through the
 * include order (-I shim -I- -I reference), which is exactly the drop-in:
 * the integrator's source is not touched.  The GPU test compares the result
 * with the CPU oracle.
 */
#include <cstring>

#include "GridMPI.h"
#include "GPUlab.h"
#include "BoundaryConditions.h"
#include "ArgumentParser.h"
#include "LSRK3_IntegratorMPI.h"

/* A lab in the style of the reference's GPUlab* cases (e.g. GPUlabSICCloud,
 * Sim_SICCloudMPI.h:309-325): every SKIN face gets its boundary condition
 * from BoundaryConditions<GridMPI>. */
class DriverLab : public GPUlab
{
    int m_refl[6];

protected:
    void _apply_bc(const double t = 0)
    {
        BoundaryConditions<GridMPI> bc(grid.pdata());
        if (myFeature[0] == SKIN) { if (m_refl[0]) bc.template applyBC_reflecting<0,0,ghostmap::X>(halox.left);  else bc.template applyBC_absorbing<0,0,ghostmap::X>(halox.left); }
        if (myFeature[1] == SKIN) { if (m_refl[1]) bc.template applyBC_reflecting<0,1,ghostmap::X>(halox.right); else bc.template applyBC_absorbing<0,1,ghostmap::X>(halox.right); }
        if (myFeature[2] == SKIN) { if (m_refl[2]) bc.template applyBC_reflecting<1,0,ghostmap::Y>(haloy.left);  else bc.template applyBC_absorbing<1,0,ghostmap::Y>(haloy.left); }
        if (myFeature[3] == SKIN) { if (m_refl[3]) bc.template applyBC_reflecting<1,1,ghostmap::Y>(haloy.right); else bc.template applyBC_absorbing<1,1,ghostmap::Y>(haloy.right); }
        if (myFeature[4] == SKIN) { if (m_refl[4]) bc.template applyBC_reflecting<2,0,ghostmap::Z>(haloz.left);  else bc.template applyBC_absorbing<2,0,ghostmap::Z>(haloz.left); }
        if (myFeature[5] == SKIN) { if (m_refl[5]) bc.template applyBC_reflecting<2,1,ghostmap::Z>(haloz.right); else bc.template applyBC_absorbing<2,1,ghostmap::Z>(haloz.right); }
    }

public:
    DriverLab(GridMPI& g, const uint_t nslices, const int* bc) : GPUlab(g, nslices, 0)
    {
        for (int i = 0; i < 6; ++i) m_refl[i] = bc ? bc[i] : 0;
    }
};

extern "C" int drv_dims(int* d)
{
    d[0] = GridMPI::sizeX; d[1] = GridMPI::sizeY; d[2] = GridMPI::sizeZ;
    return 0;
}

/* nsteps LSRK3 steps of LSRK3_IntegratorMPI::operator() from (U, R), in
 * place.  sos_cpp selects the reference's -SOSkernel cpp (CPU sound speed on
 * the host state) instead of cuda.  host_sync = 0 keeps the state on the
 * device between stages (then -SOSkernel must be cuda).  Returns the last dt. */
extern "C" double drv_run_sliced(int nsteps, double cfl, int sos_cpp, const int* bc, float** U, float** R, int host_sync,
                                 int nslices);

extern "C" double drv_run(int nsteps, double cfl, int sos_cpp, const int* bc, float** U, float** R, int host_sync)
{
    return drv_run_sliced(nsteps, cfl, sos_cpp, bc, U, R, host_sync, (int)GridMPI::sizeZ);
}

/* The same with the lab built for chunks of nslices planes (the reference's
 * GPUlab(grid, nslices)); with MPCF_GPULAB_WINDOW=1 in the environment the
 * lab streams the block through device slots chunk by chunk. */
extern "C" double drv_run_sliced(int nsteps, double cfl, int sos_cpp, const int* bc, float** U, float** R, int host_sync,
                                 int nslices)
{
    const size_t n = (size_t)GridMPI::sizeX * GridMPI::sizeY * GridMPI::sizeZ;
    GridMPI grid(1, 1, 1);
    for (int q = 0; q < 7; ++q)
    {
        std::memcpy(grid.pdata()[q], U[q], sizeof(float) * n);
        std::memcpy(grid.ptmp()[q], R[q], sizeof(float) * n);
    }
    DriverLab lab(grid, (uint_t)nslices, bc);
    lab.set_host_sync(host_sync != 0);
    const char* argv[] = {"drv", "-verb", "0", "-SOSkernel", sos_cpp ? "cpp" : "cuda"};
    ArgumentParser parser(5, argv);
    LSRK3_IntegratorMPI stepper(&grid, &lab, cfl, parser);
    double dt = 0;
    for (int s = 0; s < nsteps; ++s) dt = stepper(1e30);
    if (!host_sync) lab.download();
    for (int q = 0; q < 7; ++q)
    {
        std::memcpy(U[q], grid.pdata()[q], sizeof(float) * n);
        std::memcpy(R[q], grid.ptmp()[q], sizeof(float) * n);
    }
    return dt;
}
