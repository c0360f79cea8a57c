// GPUlab.h -- the reference's lab interface (source/GPUlab.h:33-265) on the
// B200 path: same constructor, same public members, same protected hooks
// (myFeature, grid, halox/haloy/haloz, virtual _apply_bc), so the
// reference's LSRK3_IntegratorMPI and GPUlab* subclasses compile against
// it unchanged.
//
// Behaviour: the block lives on the device in a libmpcf_b200 solver; one
// process_all is one fused stage kernel (ghosts from the recorded boundary
// conditions, WENO5/HLLC fluxes in x/y/z, divergence, register and state
// update).  `nslices` is accepted and checked like the reference
// (GPUlab.cpp:37-47).  A block that fits on the device is not chunked.  A
// block that does not (or any block with MPCF_GPULAB_WINDOW=1 and nslices <
// sizeZ) runs windowed as the reference runs it: process_all and max_sos
// stream grid.pdata()/ptmp() through MPCF_GPULAB_SLOTS (default 6) device
// slots in chunks of nslices planes (mpcf_create_window, mpcf_window_stage,
// mpcf_window_max_sos), the host copy always current.  With host synchronisation on
// (the default) the observable contract of the reference holds: max_sos
// and process_all read grid.pdata()/ptmp() and process_all leaves the new
// state in grid.pdata() and the new register in grid.ptmp()
// (GPUlab.cpp:772-788).  set_host_sync(false) keeps the data on the device
// between calls (no PCIe traffic per stage); download() then refreshes the
// host copy on demand.
#pragma once

#include <mpi.h>
#include <string>
#include <vector>

#include "Types.h"
#include "GridMPI.h"
#include "GPU.h"
#include "BoundaryConditions.h"

struct mpcf_solver;

class GPUlab
{
public:
    static const uint_t sizeX = GridMPI::sizeX;
    static const uint_t sizeY = GridMPI::sizeY;
    static const uint_t sizeZ = GridMPI::sizeZ;
    static const uint_t SLICE_GPU = GridMPI::sizeX * GridMPI::sizeY;

    GPUlab(GridMPI& G, const uint_t nslices, const int verbosity = 0);
    virtual ~GPUlab();

    void load_ghosts(const double t = 0);
    double max_sos(float& sos);
    double process_all(const Real a, const Real b, const Real dtinvh);

    // info (GPUlab.h:260-264): one chunk covers a device-resident block
    inline uint_t number_of_chunks() const { return m_window ? sizeZ / nslices : 1; }
    inline uint_t chunk_slices() const { return m_window ? nslices : sizeZ; }
    inline uint_t chunk_start_iz() const { return 0; }
    inline uint_t chunk_id() const { return 1; }

    // B200 additions
    mpcf_solver* solver() const { return m_solver; }
    bool windowed() const { return m_window; }
    void set_host_sync(const bool on) { m_host_sync = on || m_window; }
    bool host_sync() const { return m_host_sync; }
    void upload();      // grid.pdata()/ptmp() -> device
    void download();    // device -> grid.pdata()/ptmp()
    void face_bc(int bc[6]) const { for (int i = 0; i < 6; ++i) bc[i] = m_bc[i]; }

    // called by BoundaryConditions (one face of the lab that owns `halo`)
    void record_bc_face(const int face, const int type);

protected:
    enum { SKIN, FLESH } myFeature[6];
    GridMPI& grid;

    // The ghosts are synthesised on the device from the recorded boundary
    // conditions, so the halo buffers are never read.  They still hold
    // storage in the reference's layout (NVAR arrays of Nhalo per side),
    // filled with a marker: a subclass whose _apply_bc writes them by hand
    // (a condition BoundaryConditions cannot express) is detected by
    // load_ghosts instead of being ignored.
    struct Halo
    {
        static const uint_t NVAR = GridMPI::NVAR;
        const uint_t Nhalo;
        std::vector<Real> store;
        RealPtrVec_t left, right;
        Halo(const uint_t sizeHalo);
        bool untouched() const;   // every value still the marker
    };
    Halo halox, haloy, haloz;

    // boundary conditions (applied for myFeature == SKIN)
    virtual void _apply_bc(const double t = 0) {}

private:
    const uint_t nslices;
    int m_verbosity;
    mpcf_solver* m_solver;
    int m_bc[6];
    bool m_bc_dirty;
    bool m_host_sync;
    long m_ghost_calls;     // load_ghosts calls so far
    bool m_check_halos;     // check the halos after every _apply_bc, not only the first
    bool m_window;          // the block streams through device slots in nslices chunks
};
