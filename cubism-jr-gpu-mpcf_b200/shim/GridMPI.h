// GridMPI.h -- the block plus its place in the Cartesian process grid
// (source/GridMPI.h:26-145), single GPU: the hot path runs on one rank, so
// the topology is 1x1x1 and every face is a physical boundary.
#pragma once

#include <mpi.h>
#include <cstdio>
#include <cstdlib>
#include "NodeBlock.h"

class GridMPI : public NodeBlock
{
protected:
    int myrank, mypeindex[3], pesize[3];
    int nbrrank[6];
    double gextent[3];
    MPI_Comm cart_world;

public:
    GridMPI(const int npeX = 1, const int npeY = 1, const int npeZ = 1, const double maxextent = 1)
        : NodeBlock()
    {
        NodeBlock::clear();
        pesize[0] = npeX; pesize[1] = npeY; pesize[2] = npeZ;
        int world = 1;
        MPI_Comm_size(MPI_COMM_WORLD, &world);
        if (npeX * npeY * npeZ != world || world != 1)
        {
            fprintf(stderr, "[GridMPI ERROR: the B200 hot path runs one domain per process (got %dx%dx%d ranks)]\n", npeX, npeY, npeZ);
            exit(1);
        }
        const int blocks[3] = {sizeX, sizeY, sizeZ};
        const int periodic[3] = {1, 1, 1};
        h = maxextent / std::max(pesize[0] * sizeX, std::max(pesize[1] * sizeY, pesize[2] * sizeZ));
        MPI_Cart_create(MPI_COMM_WORLD, 3, pesize, periodic, 1, &cart_world);
        MPI_Comm_rank(cart_world, &myrank);
        MPI_Cart_coords(cart_world, myrank, 3, mypeindex);
        for (int i = 0; i < 6; ++i) nbrrank[i] = myrank;
        for (int i = 0; i < 3; ++i)
        {
            extent[i] = h * blocks[i];
            gextent[i] = extent[i] * pesize[i];
        }
    }

    void peindex(int mypeindex_[3]) const { for (int i = 0; i < 3; ++i) mypeindex_[i] = mypeindex[i]; }
    void getNeighborRanks(int nbr[6]) const { for (int i = 0; i < 6; ++i) nbr[i] = nbrrank[i]; }
    int getBlocksPerDimension(int d) const { return pesize[d]; }
    bool isroot() const { return myrank == 0; }
    MPI_Comm getCartComm() const { return cart_world; }
    double getH() const { return h; }
    void getGlobalExtent(double g[3]) const { g[0] = gextent[0]; g[1] = gextent[1]; g[2] = gextent[2]; }
};
