// Internal declarations shared by the spgnb translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <utility>
#include <set>
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
void count_launches(long long n);  // kernels of a replayed graph; negative to undo captured ones
unsigned long long launches_so_far();
bool sync_check();

#define SPGNB_CHECK_LAUNCH(name)                                        \
    do                                                                  \
    {                                                                   \
        ::spgnb::count_launch();                                        \
        cudaError_t e__ = cudaGetLastError();                           \
        if (e__ == cudaSuccess && ::spgnb::sync_check()) e__ = cudaDeviceSynchronize(); \
        if (e__ != cudaSuccess) return ::spgnb::cuda_fail(e__, name);   \
    } while (0)

// The force pass's kernels (slot pack, pruning, pair kernel, finishing pass,
// and the soft-core and long-range kernels around it) are launched as
// programmatic dependents of the kernel before them on the
// stream: a grid may be scheduled while its predecessor drains, and each of
// them starts with grid_dep_wait(), which returns once the predecessor has
// completed and its writes are visible.  Every thread of these kernels passes
// that wait before anything else, so a grid never completes before its
// predecessor and the chain stays ordered.  Inside a stream capture (the
// batched engine's graphs) they are launched plainly.
template <typename... KArgs, typename... Args>
cudaError_t launch_dependent(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                             Args&&... args)
{
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess)
    {
        // not known: launch plainly, and leave no error behind for the
        // launch check that follows
        cudaGetLastError();
        cs = cudaStreamCaptureStatusActive;
    }
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = cs == cudaStreamCaptureStatusNone ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Waits for the grid launched before this one on the stream (a programmatic
// dependent launch) to complete with its writes visible; a no-op when the
// grid was launched plainly.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

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
constexpr int kChunk = 32;            // table elements a search warp stages before writing
constexpr int kMaxStencil = 192;      // MAX_GRID_NEIGHBORS of neighbor_list.cpp:3
constexpr int kMaxCellAtoms = 2048;   // hard per-cell capacity of the in-cell sort
constexpr double kForceScale = 4294967296.0;   // 2^32 per kcal/mol/A
constexpr double kForceUnscale = 1.0 / 4294967296.0;
constexpr double kEnergyScale = 4294967296.0;  // totals in 2^-32 kcal/mol
constexpr float kPadCoordinate = 1.0e4f;

// device counters (int slots of NL::d_counters)
enum Counter
{
    kCntClusters = 0,   // (unused)
    kCntItems = 1,
    kCntEntries = 2,    // 64-bit: neighbour-table elements of the last build (slots 2,3)
    kCntOverflow = 4,   // bit flags
    kCntNeed = 5,       // some system rebuilds in the current update
    kCntBuilds = 6,
    kCntMaxCell = 7,
    kCntWords = 8,      // 64-bit: listed partners summed over atoms, last build (slots 8,9)
    kCntNbr = 10,       // (unused)
    kCntPrune = 11,     // some system's pruned lists must be redone before the next force
    kCntPruneDone = 12, // blocks of the running prune kernel that finished
    kCntPrunes = 13,    // prunings performed
    kCntPWords = 14,    // 64-bit: words of the running pruning (slots 14,15)
    kCntPWordsLast = 16,  // 64-bit: words of the last completed pruning (slots 16,17)
    kCntPruneNext = 18,   // the next cluster a warp of the running prune kernel takes
    kCntSearchNext = 19,  // the next cluster a warp of the running search kernel takes
    kCntPairNext = 20,    // the next cluster a warp of the running force kernel takes
    kCntPairDone = 21,    // blocks of the running force kernel that finished
    kCntSize = 24
};

enum OverflowBits
{
    kOvfList = 1,      // neighbour count above max_neighbor_numbers (export)
    kOvfGrid = 2,      // cell above max_atom_in_grid_numbers
    kOvfPairs = 4,     // a neighbour table above its capacity
    kOvfCellHard = 8,  // cell above the in-cell sort capacity
    kOvfStencil = 16,
    kOvfTable = 32,    // (unused)
    kOvfWords = 64     // a pruned per-atom list above its capacity
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

// One periodic system of a list: geometry of its reference grid and the
// ranges it owns in the concatenated atom and cell arrays.
struct SysDesc
{
    Cell cell, rcell;
    float gl, cs2, list_radius;
    float frac_norm[3];
    int Nx, Ny, Nz, cell_begin;
    int cl_begin, cl_cap;   // the system's fixed range of clusters
    int atom_begin, atom_count, triclinic;
    int all_safe;   // every cluster pair the search can meet is inside half a box: one image per pair
    float prune_r2; // squared radius of the pruned lists, (cutoff + buffer)^2; huge when pruning is off
    float permit2;  // squared displacement that triggers a rebuild (skin * skin_permit)^2
    Cell qcell;     // cell / 2^22: Cartesian length of one step of the 22-bit cluster centres
};

// Pair-function parameters of one system.
struct ForceParams
{
    float rc2, beta, beta3, w_scale;
    int use_fit, n_types, table_begin, t4_begin;  // t4_begin: first element of the system's T^3 table
};

constexpr int kMaxSlots = 1 << 23;   // slots of one list (int offsets into the per-slot regions)
constexpr int kMaxSystemSlots = 1 << 22;  // slots of one system: the partner field of a pruned-list word
constexpr int kMaxTypes = 128;       // LJ type field (7 bits) of a slot's aux record

}  // namespace spgnb

// ----------------------------------------------------------- host handles
// First-fit allocator of index ranges in [0, cap), for the pool of systems.
struct RangePool
{
    long long cap = 0;
    std::map<long long, long long> free_;  // begin -> length
    void reset(long long c)
    {
        cap = c;
        free_.clear();
        if (c > 0) free_[0] = c;
    }
    // first range of n indices, or -1 (n = 0 is an empty range at 0)
    long long alloc(long long n)
    {
        if (n <= 0) return 0;
        for (auto it = free_.begin(); it != free_.end(); ++it)
            if (it->second >= n)
            {
                const long long b = it->first, len = it->second;
                free_.erase(it);
                if (len > n) free_[b + n] = len - n;
                return b;
            }
        return -1;
    }
    void release(long long b, long long n)
    {
        if (n <= 0) return;
        auto it = free_.emplace(b, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first)
        {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin())
        {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first)
            {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
    long long available() const
    {
        long long t = 0;
        for (const auto& f : free_) t += f.second;
        return t;
    }
};

struct SysHost
{
    int atom_begin = 0, atom_count = 0;
    spgnb_ltmatrix3 cell{}, rcell{};
    float cutoff = 0, skin = 0, gl = 0, cs2 = 0;
    int dims[3] = {0, 0, 0};
    int cell_begin = 0;     // cells [cell_begin, cell_begin + G]; the extra one ends the run table
    int cl_begin = 0, cl_cap = 0;
    long long run_begin = 0, run_count = 0;
    bool triclinic = false;
    int cells() const { return dims[0] * dims[1] * dims[2]; }
};

// A neighbour list over one or more independent periodic systems.  Every
// system owns ranges of the atom, cell, cluster and run arrays; ranges no
// system owns map to the parking descriptor (index S), which never rebuilds
// or prunes.  The C ABI's NEIGHBOR_LIST is the one-system case; the batched
// engine uses many, admitted and retired while the others run.
struct spgnb_nl
{
    int S = 1;             // system ids [0, S); descriptor S parks unused ranges
    std::vector<SysHost> sys;
    std::vector<char> live;
    std::set<int> free_ids;
    RangePool cell_pool, cl_pool, run_pool;
    long long runs_cap = 0;
    int n_cap = 0;         // atoms, all systems
    int G = 0;             // cells, all systems
    float cutoff = 0, skin = 0, grid_length = 0, cs2 = 0;   // system 0 (one-system API)
    int dims[3] = {0, 0, 0};
    spgnb_ltmatrix3 cell{}, rcell{};
    bool triclinic = false;
    spgnb_nl_options opt{};
    int clusters_cap = 0;
    int table_cap = 0;     // neighbour-table elements per cluster
    int list_cap = 0;      // words reserved per cluster for its pruned partner list (a multiple of 32)
    float prune_rc = 0;    // cutoff the pruned lists are made for
    bool built = false;
    int local_atoms = 0;
    // neighbour tables one-sided (J >= I), except for the clusters holding an
    // atom flagged in two_sided_atoms (the soft-core kernel's perturbed
    // atoms) and after nl_symmetrize (every cluster two-sided, until the next
    // build); what the last build made, and its exclusion arrays
    mutable bool sym_built = false;
    // reverse index of the tables: for each cluster J, the elements
    // c * table_cap + t of the lower clusters' tables (c < J) that hold J,
    // ascending; with the cluster's own elements J' >= J it gives every atom
    // its partners on both sides (the exports) from one-sided tables
    int* d_rev = nullptr;        // clusters_cap x table_cap
    int* d_rev_count = nullptr;  // clusters_cap
    mutable bool rev_built = false;  // made from the current tables
    mutable const unsigned char* two_sided_atoms = nullptr;
    mutable const unsigned char* two_sided_built = nullptr;
    const int *ex_start_last = nullptr, *ex_list_last = nullptr, *ex_num_last = nullptr;

    std::vector<spgnb::SysDesc> h_desc;  // host copy of d_sys
    spgnb::SysDesc* d_sys = nullptr;
    int* d_atom_sys = nullptr;    // system of each atom
    int* d_cell_sys = nullptr;    // system of each cell
    // grid
    int* d_run_start = nullptr;   // G+1: candidate runs of each cell
    int2* d_runs = nullptr;       // {first cell | stencil flags << 28, last cell + 1}
    int* d_cell_count = nullptr;  // G
    int* d_cell_cursor = nullptr; // G
    int2* d_cell_cl = nullptr;    // G: the cell's clusters [x, y)
    // per system: rebuild and prune requests, clusters of the last build
    int* d_live = nullptr;
    int* d_need = nullptr;
    int* d_prune = nullptr;
    int* d_ncl = nullptr;
    // per atom
    int* d_atom_cell = nullptr;
    int* d_atom_shift = nullptr;  // packed lattice shift used by the wrap
    int* d_tmp_atoms = nullptr;   // slots_cap
    float4* d_wrapped = nullptr;  // brick-wrapped coordinates of the last binning
    int* d_atom_slot = nullptr;   // slot of each atom in the last build
    // per slot
    int* d_slot_atom = nullptr;
    float4* d_slot_x0 = nullptr;  // raw coordinates at the build, w = global index
    int* d_slot_gid = nullptr;    // the same global index, compact (-1: empty slot)
    float4* d_slot_d0 = nullptr;  // offset from the cluster centre at the build
    int2* d_slot_ex = nullptr;    // first and last entry of the atom's exclusion list
    int* d_slot_count = nullptr;  // full-list length of each slot
    // per cluster
    int* d_cl_cell = nullptr;
    int* d_cl_sys = nullptr;
    uint4* d_cl_u = nullptr;      // fractional centre (2^32 per box vector), w = radius bits
    int4* d_cl_q = nullptr;       // the same centre as 22-bit integers (2^22 per box vector)
    float4* d_cl_c = nullptr;     // half extents of the cluster's bounding box about its centre, w = radius
    // neighbour tables: every cluster sharing a listed pair with this one, in
    // search order, table_cap elements reserved per cluster
    int* d_tcount = nullptr;      // elements of each cluster's table
    float4* d_tab = nullptr;      // {D = centre difference (minimum image), neighbour slot base | image flag << 30}
    uint2* d_tmask = nullptr;     // 64-bit pair mask: bit a*8 + b = own slot a with neighbour slot b
    // pruned per-cluster partner lists (the half list: partners in clusters
    // J > I, and within I the pairs a < b), list_cap words reserved per
    // cluster: {partner slot | atom mask << 22 | image flag << 30}, padded to
    // 32-word windows; the length at d_pcount[8c] (a cluster near the start
    // of a periodic box can hold nearly its whole neighbourhood, so the
    // reserve is sized for that)
    unsigned* d_pwords = nullptr;
    int* d_pcount = nullptr;
    long long* d_facc = nullptr;  // per slot: the half-list kernel's int64 force sums (3), cleared after use
    // owned energy/virial sums of the per-atom mode, 8 per slot, cleared after
    // use; quantity-major (sum q of slot s at q * slot capacity + s), so the
    // lanes' adds of one quantity for consecutive partner slots share lines
    long long* d_oacc = nullptr;
    float4* d_pref = nullptr;     // slot offsets at the last pruning
    int* d_counters = nullptr;
    // reference-layout export
    spgnb_atom_group* d_nl = nullptr;
    int* d_temp = nullptr;
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
    float4* d_t4 = nullptr;          // T^3 table: {-A(a,j), -A(b,j), B(a,j), B(b,j)} at (a*T + b)*T + j
    float* d_lj_energy_atom = nullptr;
    long long* d_frc_acc = nullptr;  // 4 x int64 per local atom (reference-layout path)
    long long* d_totals = nullptr;   // 8 x int64 fixed point
    long long* d_excl_total = nullptr;  // PME excluded-pair correction energy, int64 fixed point
    int2* d_xs_sn = nullptr;            // symmetric exclusion CSR of the fused correction (local indices):
    int* d_xs_list = nullptr;           //   {first entry, count} per atom, the partners
    bool xs_on = false;
    float4* d_pos = nullptr;         // per slot (spgnb list) or per atom (atom-group path)
    int* d_pos_type = nullptr;
    int pos_cap = 0;
    float4* d_sdata = nullptr;       // spgnb list: per-step slot offsets and charges (+ the null slot)
    int4* d_slot_aux = nullptr;      // per slot: {centre x | LJ type << 22, centre y, centre z, global index}
    int sdata_cap = 0;
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

namespace spgnb
{
// Exclusive scan of value(0..n-1), handed to store(c, prefix), by one block (a multiple
// of 32 threads, each taking a contiguous chunk); the total is returned to
// every thread.
template <typename T, typename F, typename S>
__device__ __forceinline__ T block_scan_to(int n, F value, S store)
{
    __shared__ T warp_sums[32];
    const int threads = blockDim.x;
    const int per = (n + threads - 1) / threads;
    const int lo = min(n, threadIdx.x * per);
    const int hi = min(n, lo + per);
    T sum = 0;
    for (int c = lo; c < hi; c++) sum += value(c);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T v = sum;
    for (int o = 1; o < 32; o <<= 1)
    {
        const T t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    if (lane == 31) warp_sums[warp] = v;
    __syncthreads();
    const int nw = threads >> 5;
    if (warp == 0)
    {
        T w = lane < nw ? warp_sums[lane] : 0;
        for (int o = 1; o < 32; o <<= 1)
        {
            const T t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        if (lane < nw) warp_sums[lane] = w;
    }
    __syncthreads();
    T excl = v - sum + (warp > 0 ? warp_sums[warp - 1] : 0);
    for (int c = lo; c < hi; c++)
    {
        store(c, excl);
        excl += value(c);
    }
    const T total = warp_sums[nw - 1];
    __syncthreads();
    return total;
}

template <typename T, typename F>
__device__ __forceinline__ T block_scan(int n, F value, T* out)
{
    return block_scan_to<T>(n, value, [&](int c, T v) { out[c] = v; });
}


struct OwnerMap
{
    const int* atom_local;   // global index of each local atom
    int solvent_start;       // first local atom of the water tail (n when none)
    int water_points;
    __device__ __forceinline__ int remap(int a) const
    {
        return a >= solvent_start ? solvent_start + ((a - solvent_start) / water_points) * water_points : a;
    }
};

struct PerAtomOut
{
    float* energy;       // caller's atom_energy (+=)
    float* lj_energy;    // module's per-atom LJ energy
    float* direct;       // atom_direct_pme_energy
    float* virial;       // caller's LTMatrix3 array (+=), 6 floats per atom
};

// PME's excluded-pair correction fused into the pair kernel: each atom's
// excluded partners on both sides (a symmetric CSR in local indices), walked
// by the atom's warp after its list.  list == nullptr: off.
struct ExclFuse
{
    const int2* sn = nullptr;          // per local atom {first entry, count}
    const int* list = nullptr;
    const float3* crd = nullptr;       // per local atom
    const float* charge = nullptr;
    const int* atom_local = nullptr;   // global index of each local atom (the energy owner rule)
    float beta = 0.0f, beta3 = 0.0f;
    long long* total = nullptr;        // energy total, int64 fixed point (energy modes)
    float* energy = nullptr;           // per-atom energy (+=), per-atom mode
    float* virial = nullptr;           // per-atom virial (+=), per-atom mode
};

// One force evaluation over an spgnb list: slot pack (with the per-system
// prune trigger), pruning when due, and the pruned-list force kernel.
struct ForceInputs
{
    spgnb_nl* nl = nullptr;
    const float3* crd = nullptr;       // per atom, the list's atom order
    const float* charge = nullptr;
    const int* atom_type = nullptr;    // into the LJ table
    float4* slot_pos = nullptr;        // scratch, slots + 1
    int4* slot_aux = nullptr;          // scratch, slots + 1
    ForceParams p0{};                  // the one system's parameters (d_fps null)
    const ForceParams* d_fps = nullptr;  // per system (several systems)
    bool fit = true;                   // every system inside the rational fits' range
    const float4* t4 = nullptr;        // the T^3 pair tables (coefficient_table)
    int max_types = 0;                 // most types of any system's table (0: p0.n_types)
    float3* frc = nullptr;             // += forces
    long long* totals = nullptr;       // 8 fixed-point sums per system (mode >= 1)
    const int* only = nullptr;         // per-system flags: evaluate these systems only (null: all)
    int mode = 0;                      // 0 forces, 1 + totals, 2 + per-atom outputs
    int pair_blocks_per_sm = 0;        // force kernel grid: 0 = as many as are resident
    int prune_blocks_per_sm = 0;       // pruning kernel grid: 0 = 5
    OwnerMap om{nullptr, 0, 3};
    PerAtomOut pa{nullptr, nullptr, nullptr, nullptr};
    ExclFuse xf{};                     // one system only
    // cleared by the slot pack before the pair kernel runs: 8 totals, one
    // more int64, and two float arrays of n entries (any may be null)
    struct
    {
        long long* totals = nullptr;
        long long* one = nullptr;
        float* a = nullptr;
        float* b = nullptr;
        int n = 0;
    } clear;
};
int force_pipeline(const ForceInputs& in, cudaStream_t s);
// The pipeline's stages, for callers that place them themselves (the
// batched step): argument checks, the slot pack (gated on *gate when given),
// the pruning (runs for the systems flagged), the pair kernel (forces into
// the list's int64 staging, d_facc, which the finishing pass or the caller
// turns into float forces and clears).
int force_check(const ForceInputs& in);
int launch_pack(const ForceInputs& in, cudaStream_t s, const int* gate);
int launch_prune(const ForceInputs& in, cudaStream_t s);
int launch_pair_kernel(const ForceInputs& in, cudaStream_t s);
// The force kernel's coefficient table of a T x T square pair table {A, B}:
// element (a*T + b)*T + j = {-A_aj, -A_bj, B_aj, B_bj}, the rows of an atom
// pair (a, b) of a cluster against every partner type j.
std::vector<float4> coefficient_table(const float2* table, int T);
// coefficient_table uploaded to a new device array (freeing the old one).
int build_t4(const float2* table, int T, float4** d_t4);
// Adds the module's int64 force accumulators of atoms [0, n) to frc and
// clears them (the reference-layout and correction paths end with it).
int lj_finalize_forces(spgnb_lj* lj, int n, float3* frc, cudaStream_t s);

// Neighbour-list internals shared with the force and batch code.
int nl_create_multi(int n_systems, const int* atom_counts, const spgnb_ltmatrix3* cells,
                    const spgnb_ltmatrix3* rcells, const float* cutoffs, const float* skins,
                    const spgnb_nl_options* opt, spgnb_nl** out);
// Host-to-device uploads from one pinned staging buffer, so the copies are
// asynchronous: the caller keeps the buffer until an event recorded after
// them has completed.  Without a buffer the copies read the caller's memory
// directly (pageable: the copy completes before the call returns).
struct PinnedStage
{
    char* p = nullptr;
    size_t cap = 0, used = 0;
    cudaEvent_t ev = nullptr;
    bool busy = false;
};
struct Uploader
{
    PinnedStage* st = nullptr;
    int put(void* dst, const void* src, size_t bytes, cudaStream_t s);
};

// Capacities of an empty pool of systems.
struct NLPoolSpec
{
    int systems = 0;
    int atoms = 0;
    int cells = 0;        // including one extra cell per system
    int clusters = 0;
    long long runs = 0;
    int table_cap = 0;    // neighbour-table elements per cluster
    int list_cap = 0;     // pruned-list words per cluster
    float prune_rc = 0;   // the largest cutoff
};
int nl_create_pool(const NLPoolSpec& spec, const spgnb_nl_options* opt, spgnb_nl** out);
// Fills a system's grid geometry from its box, cutoff and skin; checks them.
int nl_init_system(SysHost& sh, int atom_count, spgnb_ltmatrix3 cell, spgnb_ltmatrix3 rcell, float cutoff,
                   float skin, int index);
// Candidate-cell runs of a system with cell ids from 0: run_start has G + 1
// entries.
int nl_system_runs(const SysHost& sh, std::vector<int>& run_start, std::vector<int2>& runs);
// Table and pruned-list capacities for a system of this density and cutoff.
// Words reserved per cluster for a pruned list of per_cluster partners
// (with a margin and room for the padding to whole windows).
int list_cap_for(double per_cluster);
void nl_capacity_for(double atoms_per_A3, double atom_count, float cutoff, float skin, float prune_buffer,
                     double* table_per_cluster, double* words_per_cluster);
// Takes a free system id and the cell, cluster and run ranges of a system
// whose atoms occupy [sh.atom_begin, + sh.atom_count); SPGNB_E_OOM (no
// message) when the pool has no room now.  The system rebuilds when the
// caller sets its flag for a kBuildPreset update.
int nl_admit(spgnb_nl* nl, SysHost sh, const std::vector<int>* run_start, const std::vector<int2>* runs,
             cudaStream_t s, int* id, Uploader up = Uploader{});
// Bytes an Uploader needs for a system's list data (runs, run table, descriptor).
size_t nl_admit_upload_bytes(const SysHost& sh, size_t n_runs);
// Returns a system's ranges to the pool; its atoms map to the parking descriptor.
int nl_retire(spgnb_nl* nl, int id, cudaStream_t s);
// Every live system re-prunes before the next force evaluation.
int nl_prune_all(spgnb_nl* nl, cudaStream_t s);
// Makes the last build's neighbour tables two-sided: re-runs its search (same
// clusters and build coordinates, so the same list) when they are one-sided.
int nl_symmetrize(const spgnb_nl* nl, cudaStream_t s);
// Makes the tables of the clusters holding a flagged atom (per local atom,
// non-zero) two-sided, in the last build (re-searched if needed) and the
// later ones.
int nl_two_sided_atoms(const spgnb_nl* nl, const unsigned char* d_flags, cudaStream_t s);
enum BuildHow
{
    kBuildSkin = 0,
    kBuildForced = 1,
    kBuildInterval = 2,
    kBuildPreset = 3
};
// aux: kBuildInterval - per-system steps done; kBuildPreset - per-system
// flags of the systems to rebuild.  active (optional): per system, 0 = frozen
// (no forced or interval rebuild).
int nl_queue_build(spgnb_nl* nl, int n, const float3* d_crd, const int* d_atom_local, const int* ex_start,
                   const int* ex_list, const int* ex_num, int how, cudaStream_t s, const int* d_aux = nullptr,
                   int interval = 0, const int* d_active = nullptr);
// The build without the decision: the caller has set the per-system need
// flags and the counters' rebuild flag (every kernel returns at once when
// that flag is zero).
int nl_queue_build_body(spgnb_nl* nl, int n, const float3* d_crd, const int* d_atom_local, const int* ex_start,
                        const int* ex_list, const int* ex_num, cudaStream_t s);
int nl_regrow(spgnb_nl* nl, int flags);
int nl_set_prune_rc(spgnb_nl* nl, float rc, cudaStream_t s);
size_t nl_device_bytes(const spgnb_nl* nl);

}  // namespace spgnb
