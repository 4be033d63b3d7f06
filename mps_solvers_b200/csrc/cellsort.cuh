// cellsort.cuh -- the neighbour-search rebuild (the reference's divideCell).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "mps_device.cuh"

namespace mpsb {

constexpr int SORT_THREADS = 256;
constexpr int SORT_ITEMS = 8;
constexpr int SORT_TILE = SORT_THREADS * SORT_ITEMS;  // 2048 keys per tile
constexpr int SORT_RADIX = 256;
constexpr uint32_t SORT_FUSED_SCAN_TILES = 64;  // up to this many tiles the downsweep scans the histograms (measured: faster at 35, slower at 152)

inline uint32_t sort_tiles(uint32_t cap) { return (cap + SORT_TILE - 1) / SORT_TILE; }

// Number of 8-bit passes to sort keys in [0, ncells] (ncells is the
// out-of-grid sentinel).
inline int sort_passes(uint32_t ncells) {
    int bits = 0;
    while (bits < 32 && (uint64_t(1) << bits) <= ncells) bits++;
    return (bits + 7) / 8;
}

// Scratch of one sort, sized for `cap` keys.
struct SortScratch {
    uint32_t* keys[2];
    uint32_t* vals[2];
    uint32_t* hist;  // SORT_RADIX * tiles
    uint32_t tiles;
};

// Pending particle update applied by the rebuild (the second phase of the
// reference's two-phase stages, which divideCell always follows).
enum ApplyMode : int {
    APPLY_NONE = 0,
    APPLY_SET_VEL = 1,  // fluid: u = tmp, x = x + dt*tmp      (calVisc_expl)
    APPLY_ADD_VEL = 2,  // fluid: u = u + tmp, x = x + dt*tmp  (collision, calDash)
};

// Launchers (all asynchronous on `st`).
// Stable LSD radix sort of (keys[0], vals[0]) over *n_dev keys; returns the
// buffer index (0/1) that holds the result.
int launch_radix_sort(SortScratch& s, const uint32_t* n_dev, int passes, uint32_t cap, cudaStream_t st);
// The rebuild's keys and sort: the cell key of every active particle (after
// the pending update; with batch.n > 0 g is the whole cell space and each
// particle, by id, uses its scene's grid) computed by the first pass's
// upsweep, then the sort over sc->np keys.  Returns the buffer index as
// launch_radix_sort.  The cell table is filled by the gather that follows.
int launch_keys_and_sort(const float4* pos, const float4* tmp, int apply, const Grid& g, Scalars* sc,
                         const uint32_t* id, const BatchDev& batch, SortScratch& s, int passes, cudaStream_t st);


// ---- merge rebuild
// Between two rebuilds only the particles whose cell changed move in the
// stably sorted order: the others keep their relative order (their keys are
// unchanged and they were sorted by key, then by previous position).  The
// new order is therefore the merge of the unchanged particles, in place,
// with the changed ones sorted by (new key, previous position), which is
// exactly the stable sort's result.  The keys kernel finds the changed
// particles, one block sorts them (in shared memory up to
// MERGE_SMEM_CAP of them, else in global memory, slowly but correctly), and
// the merge gather (physics.cuh) moves every particle to its merged
// position and derives the new cell table from the old one.
constexpr uint32_t MERGE_SMEM_CAP = 8192;
constexpr int MERGE_SORT_THREADS = 1024;

struct MergeScratch {
    uint32_t* newkey = nullptr;   // cap: each particle's key after the pending update
    uint32_t* changed = nullptr;  // cap: positions of the changed particles, in no order
    uint64_t* a = nullptr;        // cap: (new key << 32 | position) of the changed, ascending
    uint32_t* b = nullptr;        // cap: positions of the changed, ascending
    uint32_t* count = nullptr;    // [0] changed found by the keys kernel, [1] the count the merge uses
};

// The keys, the changed list and its two sorted orders (two launches).  The
// merge gather follows (launch_merge_gather).
void launch_merge_keys_sort(const float4* pos, const float4* tmp, int apply, const Grid& g, Scalars* sc,
                            const uint32_t* id, const BatchDev& batch, const uint32_t* cell_old,
                            const MergeScratch& m, uint32_t cap, cudaStream_t st);
cudaError_t merge_sort_setup();

// Same pieces with n given on the host (for the device-pointer primitive).
void launch_cell_keys_plain(const float4* pos, uint32_t n, const Grid& g, uint32_t* keys, uint32_t* vals,
                            cudaStream_t st);
void launch_cell_start_plain(const uint32_t* keys_sorted, uint32_t n, const Grid& g, uint32_t* cell_start,
                             uint32_t* n_in_grid, cudaStream_t st);
// exclusive scan of `total` uint32 counters in place (one block)
void launch_scan_exclusive(uint32_t* a, uint32_t total, cudaStream_t st);
void launch_cell_end_from_start(const uint32_t* cell_start, uint32_t ncells, uint32_t* start_out,
                                uint32_t* end_out, cudaStream_t st);

// cell_start[c] = first sorted position whose key is >= c, for c in
// [0, ncells]; equal to the reference's serial prefix sum of per-cell counts
// (MPS_CAL_expl_v1.0/MPS_GPU.cpp:293-297), with cell_end[c] = cell_start[c+1]
// and cell_start[ncells] = number of particles inside the grid.
__device__ __forceinline__ void cell_start_fill(const uint32_t* keys, uint32_t n, uint32_t ncells, uint32_t p,
                                                uint32_t* cell_start) {
    long long prev = p > 0 ? (long long)keys[p - 1] : -1ll;
    long long cur = p < n ? (long long)keys[p] : (long long)ncells;
    if (cur > (long long)ncells) cur = ncells;
    for (long long c = prev + 1; c <= cur; c++) cell_start[c] = p;
}


}  // namespace mpsb
