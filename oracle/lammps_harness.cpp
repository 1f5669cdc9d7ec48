// C entry points around the reference's own nnp::InterfaceLammps
// (src/libnnpif/LAMMPS/InterfaceLammps.cpp, compiled from its sources with
// libnnp into oracle/_ref/libnnplammps.so): the LAMMPS-interface oracle.
//
// TEST INFRASTRUCTURE ONLY: loaded by tests/ (through oracle/lammps_ref.py).
// The product never links or loads this library.
#include <cstdint>
#include <limits>
#include <string>
#include <vector>

#include "InterfaceLammps.h"

namespace {
thread_local std::string g_err;
}

extern "C" {

const char* nnplmp_last_error() { return g_err.c_str(); }

void* nnplmp_create(const char* dir, const char* emap, int showew, double cflength, double cfenergy,
                    double lammpsCutoff, int ntypes)
{
    try
    {
        auto* p = new nnp::InterfaceLammps();
        // showew: collect warnings (no per-warning output, no limit)
        p->initialize(dir, emap, showew != 0, false, 0, showew ? 0 : -1, cflength, cfenergy, lammpsCutoff, ntypes, 0);
        return p;
    }
    catch (std::exception const& e)
    {
        g_err = e.what();
        return nullptr;
    }
}

void nnplmp_destroy(void* p) { delete static_cast<nnp::InterfaceLammps*>(p); }

int nnplmp_set_local_atoms(void* p, int n, const int* type)
{
    try
    {
        static_cast<nnp::InterfaceLammps*>(p)->setLocalAtoms(n, type);
        return 0;
    }
    catch (std::exception const& e)
    {
        g_err = e.what();
        return 1;
    }
}

// Every neighbour of every local atom at once (the loop of
// PairHDNNP::transferNeighborList): entries [offset[i], offset[i+1]) of
// local atom i.
int nnplmp_add_neighbors(void* p, int n, const int64_t* offset, const int* j, const int* type, const double* dr,
                         const double* d2)
{
    try
    {
        auto* lmp = static_cast<nnp::InterfaceLammps*>(p);
        for (int i = 0; i < n; ++i)
            for (int64_t e = offset[i]; e < offset[i + 1]; ++e)
                lmp->addNeighbor(i, j[e], (int64_t)j[e] + 1, type[e], dr[3 * e], dr[3 * e + 1], dr[3 * e + 2], d2[e]);
        lmp->finalizeNeighborList();
        return 0;
    }
    catch (std::exception const& e)
    {
        g_err = e.what();
        return 1;
    }
}

int nnplmp_process(void* p)
{
    try
    {
        static_cast<nnp::InterfaceLammps*>(p)->process();
        return 0;
    }
    catch (std::exception const& e)
    {
        g_err = e.what();
        return 1;
    }
}

double nnplmp_energy(void* p) { return static_cast<nnp::InterfaceLammps*>(p)->getEnergy(); }

// NaN for an index the reference refuses (std::out_of_range from its atom list).
double nnplmp_atomic_energy(void* p, int i)
{
    try
    {
        return static_cast<nnp::InterfaceLammps*>(p)->getAtomicEnergy(i);
    }
    catch (std::exception const& e)
    {
        g_err = e.what();
        return std::numeric_limits<double>::quiet_NaN();
    }
}

// Adds the forces to f[nall][3] (contiguous) through LAMMPS-style row pointers.
int nnplmp_get_forces(void* p, double* f, int64_t nall)
{
    try
    {
        std::vector<double*> rows((size_t)nall);
        for (int64_t k = 0; k < nall; ++k) rows[(size_t)k] = f + 3 * k;
        static_cast<nnp::InterfaceLammps*>(p)->getForces(rows.data());
        return 0;
    }
    catch (std::exception const& e)
    {
        g_err = e.what();
        return 1;
    }
}

int64_t nnplmp_num_ew(void* p) { return (int64_t)static_cast<nnp::InterfaceLammps*>(p)->getNumExtrapolationWarnings(); }

} // extern "C"
