// Internal declarations shared by the spgnb translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "ewald_fit.h"
#include "spgnb.h"

namespace spgnb
{

// ------------------------------------------------------------------ errors
int fail(int status, const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what);
cudaStream_t stream();
int num_sms();

#define SPGNB_CUDA(call)                                               \
    do                                                                 \
    {                                                                  \
        cudaError_t e__ = (call);                                      \
        if (e__ != cudaSuccess) return ::spgnb::cuda_fail(e__, #call); \
    } while (0)

void count_launch();

#define SPGNB_CHECK_LAUNCH(name)                                        \
    do                                                                  \
    {                                                                   \
        ::spgnb::count_launch();                                        \
        cudaError_t e__ = cudaGetLastError();                           \
        if (e__ != cudaSuccess) return ::spgnb::cuda_fail(e__, name);   \
    } while (0)

// events recorded around the pair kernel when set (benchmark instrumentation)
void pair_events(cudaEvent_t* start, cudaEvent_t* stop);

template <typename T>
int dalloc(T** p, size_t count)
{
    *p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void**)p, sizeof(T) * count);
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        *p = nullptr;
        return fail(SPGNB_E_OOM, "cudaMalloc of %zu bytes failed: %s", sizeof(T) * count, cudaGetErrorString(e));
    }
    return SPGNB_OK;
}

template <typename T>
void dfree(T*& p)
{
    if (p) cudaFree((void*)p);
    p = nullptr;
}

// ---------------------------------------------------------------- constants
constexpr int kClusterSize = 8;       // atoms per cluster
constexpr int kChunk = 32;            // cluster-pair entries per work item
constexpr int kMaxStencil = 192;      // MAX_GRID_NEIGHBORS of neighbor_list.cpp:3
constexpr int kMaxCellAtoms = 2048;   // hard per-cell capacity of the in-cell sort
constexpr double kForceScale = 4294967296.0;   // 2^32 per kcal/mol/A
constexpr double kForceUnscale = 1.0 / 4294967296.0;
constexpr double kEnergyScale = 4294967296.0;  // totals in 2^-32 kcal/mol
constexpr float kPadCoordinate = 1.0e4f;

// device counters (int slots of NL::d_counters)
enum Counter
{
    kCntClusters = 0,
    kCntItems = 1,
    kCntEntries = 2,    // 64-bit counter occupies slots 2,3
    kCntOverflow = 4,   // bit flags
    kCntNeed = 5,       // rebuild requested for the current update
    kCntBuilds = 6,
    kCntMaxCell = 7,
    kCntSize = 8
};

enum OverflowBits
{
    kOvfList = 1,      // neighbour count above max_neighbor_numbers (export)
    kOvfGrid = 2,      // cell above max_atom_in_grid_numbers
    kOvfPairs = 4,     // cluster-pair list capacity
    kOvfCellHard = 8,  // cell above the in-cell sort capacity
    kOvfStencil = 16
};

// entry flags
enum EntryFlags
{
    kEntPairImage = 1  // per-pair minimum image needed (small box)
};

struct Cell
{
    float a11, a21, a22, a31, a32, a33;
};

__host__ __device__ inline Cell make_cell(const spgnb_ltmatrix3& m)
{
    return Cell{m.a11, m.a21, m.a22, m.a31, m.a32, m.a33};
}

}  // namespace spgnb

// ----------------------------------------------------------- host handles
struct spgnb_nl
{
    int n_cap = 0;
    float cutoff = 0, skin = 0, grid_length = 0, cs2 = 0;
    int dims[3] = {0, 0, 0};
    int G = 0;
    spgnb_ltmatrix3 cell{}, rcell{};
    bool triclinic = false;
    spgnb_nl_options opt{};
    int clusters_cap = 0;
    long long entries_cap = 0;
    int items_cap = 0;
    int entries_per_cluster = 0;
    bool built = false;
    int local_atoms = 0;

    // grid
    int* d_cand_start = nullptr;  // G+1
    int* d_cand = nullptr;        // cell | flags
    int* d_cell_count = nullptr;  // G
    int* d_cell_cursor = nullptr; // G
    int* d_cell_cl_start = nullptr;  // G+1 (cluster index)
    // per atom
    int* d_atom_cell = nullptr;
    int* d_atom_shift = nullptr;  // packed lattice shift used by the wrap
    int* d_tmp_atoms = nullptr;   // slots_cap
    float4* d_wrapped = nullptr;  // brick-wrapped coordinates of the last binning
    // per slot
    int* d_slot_atom = nullptr;
    float4* d_slot_x0 = nullptr;  // raw coordinates at the build
    float4* d_slot_d0 = nullptr;  // offset from the cluster centre at the build
    // per cluster
    int* d_cl_cell = nullptr;
    uint4* d_cl_u = nullptr;      // fractional centre (2^32 per box vector), w = radius bits
    float4* d_cl_c = nullptr;     // Cartesian centre (wrapped frame), w = radius
    int* d_atom_slot = nullptr;   // slot of each atom in the last build
    // cluster-pair list
    int4* d_ents = nullptr;       // {j-cluster, flags, mask bits 0-31, mask bits 32-63}
    float4* d_ents_d = nullptr;   // centre difference c_j - c_i (minimum image), Cartesian
    int4* d_items = nullptr;
    int* d_counters = nullptr;
    // reference-layout export
    spgnb_atom_group* d_nl = nullptr;
    int* d_temp = nullptr;
    // last excluded-list pointers (for exports without a rebuild)
    long long host_builds = 0;
};

struct spgnb_lj
{
    int atom_numbers = 0;
    int n_types = 0;
    float cutoff = 0;
    double long_range_factor = 0;
    double h_last_long_energy = 0;
    int* d_atom_type = nullptr;      // global types
    int* d_local_type = nullptr;     // types of local atoms (Get_Local)
    const int* d_atom_local = nullptr;  // caller's local -> global map (Get_Local)
    float2* d_table = nullptr;       // T*T square table {A, B}
    float* d_lj_energy_atom = nullptr;
    long long* d_frc_acc = nullptr;  // 4 x int64 per local atom (reference-layout path)
    long long* d_slot_acc = nullptr; // 3 x slots_cap int64, SoA by slot (cluster path)
    int slot_acc_cap = 0;
    long long* d_totals = nullptr;   // 8 x int64 fixed point
    float4* d_pos = nullptr;         // per slot (spgnb list) or per atom (atom-group path)
    int* d_pos_type = nullptr;
    int pos_cap = 0;
    int local_atoms = 0;
    bool have_energy = false, have_virial = false;
    double totals[8] = {0};
    double last_volume = 0;
};

struct spgnb_solvent
{
    spgnb_lj* lj = nullptr;
    int water_points = 3;
    int solvent_start_local = 0;     // first solvent residue
    int local_solvent_numbers = 0;
    int* d_scratch = nullptr;
};
