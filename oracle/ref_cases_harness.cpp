/*
 * ref_cases_harness.cpp -- runs the reference's own case set-ups on a host
 * grid: Sim_SteadyStateMPI (source/Sim/Sim_SteadyStateMPI.cpp:95-135),
 * Sim_SodMPI (Sim_SodMPI.cpp:20-95) and Sim_2DSBIMPI (Sim_2DSBIMPI.cpp:
 * 15-233).  TEST INFRASTRUCTURE: built by `make -C oracle ref` into
 * oracle/_ref/libref_cases.so.
 *
 * The three source files are compiled as they are, over the drop-in shim
 * (GridMPI, GPUlab, Types.h, single-rank mpi.h) and the reference's own
 * LSRK3 integrator.  Each case runs its own _setup() with -dryrun 1: that
 * builds the grid and calls the case's _ic() (and an HDF5 dump, compiled
 * out without HDF5), without allocating the GPU lab.  The 2DSBI case reads
 * its bubbles from <config>bubbles.dat in the working directory, as the
 * reference does; the caller writes it.
 */
#include <unistd.h>
#include <cstring>
#include <string>
#include <iostream>
#include <vector>
#include <cmath>
#include <algorithm>

// the reference's own headers reach these files after <iostream> and a
// namespace-std using-directive (its GPUlab.h); the shim's do not
using namespace std;

#include "Sim_SteadyStateMPI.cpp"
#include "Sim_SodMPI.cpp"
#include "Sim_2DSBIMPI.cpp"

template <class Sim>
struct CaseHarness : public Sim
{
    CaseHarness(const int argc, const char** argv) : Sim(argc, argv, 1) {}
    void setup() { this->_setup(); }
    GridMPI& grid() { return *this->mygrid; }
};

extern "C" int ref_cases_dims(int* d)
{
    d[0] = GridMPI::sizeX; d[1] = GridMPI::sizeY; d[2] = GridMPI::sizeZ;
    return 0;
}

template <class Sim>
static void run_case(const int argc, const char** argv, float** out7)
{
    CaseHarness<Sim> sim(argc, argv);
    sim.setup();
    GridMPI& g = sim.grid();
    const size_t n = (size_t)GridMPI::sizeX * GridMPI::sizeY * GridMPI::sizeZ;
    for (int q = 0; q < 7; ++q) std::memcpy(out7[q], g.pdata()[q], sizeof(float) * n);
}

/* which: 0 = SteadyState, 1 = Sod, 2 = 2DSBI.  argv[0..argc) are the case's
 * command-line options (argv[0] the program name; "-dryrun 1" is expected).
 * Runs in `workdir` and copies the 7 fields out. */
extern "C" int ref_case_ic(int which, const char* workdir, int argc, const char** argv, float** out7)
{
    char cwd[4096];
    if (!getcwd(cwd, sizeof(cwd))) return -1;
    if (chdir(workdir) != 0) return -2;
    if (which == 0)      run_case<Sim_SteadyStateMPI>(argc, argv, out7);
    else if (which == 1) run_case<Sim_SodMPI>(argc, argv, out7);
    else                 run_case<Sim_2DSBIMPI>(argc, argv, out7);
    return chdir(cwd) == 0 ? 0 : -3;
}
