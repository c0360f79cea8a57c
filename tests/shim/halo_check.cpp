// halo_check.cpp -- test harness of the drop-in shim's halo check.
//
// Two GPUlab subclasses over one block: `bc` states its boundary conditions
// through BoundaryConditions::applyBC_* (the reference's Sim_* labs do), `raw`
// writes a halo value by hand in _apply_bc, which the B200 lab cannot honour
// (its ghosts are synthesised on the device).  Usage: halo_check bc|raw.
// `bc` runs one stage and exits 0; `raw` must stop in load_ghosts with the
// lab's error message and exit status 1.
#include <cstdio>
#include <cstring>

#include "GPUlab.h"

class LabBC : public GPUlab
{
public:
    LabBC(GridMPI& G) : GPUlab(G, GridMPI::sizeZ) {}
protected:
    void _apply_bc(const double t = 0) override
    {
        BoundaryConditions<GridMPI> bc(grid.pdata());
        if (myFeature[0] == SKIN) bc.template applyBC_reflecting<0, 0, ghostmap::X>(halox.left);
        if (myFeature[1] == SKIN) bc.template applyBC_absorbing<0, 1, ghostmap::X>(halox.right);
    }
};

class LabRaw : public GPUlab
{
public:
    LabRaw(GridMPI& G) : GPUlab(G, GridMPI::sizeZ) {}
protected:
    void _apply_bc(const double t = 0) override
    {
        // an inflow condition written straight into the left x halo
        for (int q = 0; q < (int)GridMPI::NVAR; ++q) halox.left[q][0] = (Real)1;
    }
};

int main(int argc, char** argv)
{
    if (argc < 2) return 2;
    MPI_Init(&argc, &argv);
    GridMPI grid(1, 1, 1);
    for (int q = 0; q < (int)GridMPI::NVAR; ++q)
        for (size_t i = 0; i < (size_t)GridMPI::sizeX * GridMPI::sizeY * GridMPI::sizeZ; ++i)
            grid.pdata()[q][i] = q == 0 ? 1000 : (q == 4 ? 5000 : (q == 5 ? 0.18f : (q == 6 ? 4800 : 0)));
    if (!strcmp(argv[1], "bc"))
    {
        LabBC lab(grid);
        lab.load_ghosts();
        lab.process_all(0, 0.25f, 0.01f);
        printf("halo_check bc: ok\n");
    }
    else
    {
        LabRaw lab(grid);
        lab.load_ghosts();
        printf("halo_check raw: not detected\n");
    }
    MPI_Finalize();
    return 0;
}
