/*
 * ref_ic_harness.cpp -- runs the reference's own shock-induced cloud-collapse
 * initial condition on a host grid.  TEST INFRASTRUCTURE: built by
 * `make -C oracle ref` into oracle/_ref/libref_sic_ic.so.
 *
 * The reference file source/Sim/Sim_SICCloudMPI.cpp is compiled as is (its IC
 * functions are file-static, so it is included into this translation unit):
 *   post-shock state      Sim_SICCloudMPI.cpp:43-132
 *   cloud files, shapes   Sim_SICCloudMPI.cpp:134-202, Sim_SICCloudMPI.h:27-301
 *   sample, mix, Simpson  Sim_SICCloudMPI.cpp:204-357
 * It derives from Sim_SteadyStateMPI, whose source needs HDF5; the members of
 * that base the IC uses (the parser, the grid, verbosity) are set up by the
 * minimal definitions below, and the drop-in shim provides GridMPI, GPUlab,
 * Types.h (SimTools) and the single-rank mpi.h, as for the LSRK3 driver.
 * The cloud is read from cloud_config.dat and cloud.dat in the working
 * directory, as the reference does; the caller writes them.
 */
#include <unistd.h>
#include <cstring>
#include <string>
#include <iostream>
#include <vector>
#include <cmath>
#include <algorithm>

// the reference's own headers reach this file after <iostream> and a
// namespace-std using-directive (its GPUlab.h); the shim's do not
using namespace std;

#include "Sim_SICCloudMPI.cpp"

Sim_SteadyStateMPI::Sim_SteadyStateMPI(const int argc, const char** argv, const int isroot_)
    : isroot(isroot_), t(0), tend(0), tnextdump(0), dumpinterval(0), CFL(0), step(0), nsteps(0), nslices(0),
      saveinterval(0), fcount(0), verbosity(0), restart(false), dryrun(false), npex(1), npey(1), npez(1),
      mygrid(new GridMPI(1, 1, 1)), myGPU(NULL), parser(argc, argv)
{
    fname[0] = '\0';
}
void Sim_SteadyStateMPI::_setup() {}
void Sim_SteadyStateMPI::_allocGPU() {}
void Sim_SteadyStateMPI::_ic() {}
void Sim_SteadyStateMPI::_dump(const std::string) {}
void Sim_SteadyStateMPI::run() {}

struct SICHarness : public Sim_SICCloudMPI
{
    SICHarness(const int argc, const char** argv) : Sim_SICCloudMPI(argc, argv, 1) {}
    void ic() { _ic(); }
    GridMPI& grid() { return *mygrid; }
};

extern "C" int ref_sic_dims(int* d)
{
    d[0] = GridMPI::sizeX; d[1] = GridMPI::sizeY; d[2] = GridMPI::sizeZ;
    return 0;
}

/* Run Sim_SICCloudMPI::_ic() with the command-line options argv[0..argc)
 * (argv[0] is the program name) in directory `workdir` (which holds
 * cloud_config.dat and cloud.dat), with SimTools::EPSILON = eps, and copy
 * the 7 fields out.  post4 (optional) receives rho1, u1, p1, mach. */
extern "C" int ref_sic_ic(const char* workdir, int argc, const char** argv, double eps, float** out7, double* post4)
{
    char cwd[4096];
    if (!getcwd(cwd, sizeof(cwd))) return -1;
    if (chdir(workdir) != 0) return -2;
    SimTools::EPSILON = eps;
    {
        SICHarness sim(argc, argv);
        sim.ic();
        GridMPI& g = sim.grid();
        const size_t n = (size_t)GridMPI::sizeX * GridMPI::sizeY * GridMPI::sizeZ;
        for (int q = 0; q < 7; ++q) std::memcpy(out7[q], g.pdata()[q], sizeof(float) * n);
    }
    if (post4)
    {
        post4[0] = SICCloudData::rho1;
        post4[1] = SICCloudData::u1;
        post4[2] = SICCloudData::p1;
        post4[3] = SICCloudData::mach;
    }
    return chdir(cwd) == 0 ? 0 : -3;
}
