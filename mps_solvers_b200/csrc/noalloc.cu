// noalloc.cu -- mps_cell_sort_dev_noalloc: the neighbour-search rebuild
// (cell keys, stable sort by cell, cell start/end tables) without any device
// memory allocation.
//
// Why it exists: mps_cell_sort_dev allocates its scratch with cudaMalloc and
// frees it with cudaFree on every call.  Some callers cannot do that: a host
// application that hands all device memory to its own pool allocator and
// forbids any other allocation, or a latency-critical loop in which
// cudaMalloc/cudaFree (which synchronise the device) would stall other work.
// This variant keeps its scratch in one fixed device array instead, so it
// allocates nothing; the caller still provides the input positions and all
// output arrays.
//
// The array and its limits:
//   * at most MPS_NOALLOC_MAX_PARTICLES particles and MPS_NOALLOC_MAX_CELLS
//     cells per call; larger requests return MPS_ERR_CAPACITY before any
//     GPU work;
//   * the array takes 10.25 MiB on every GPU where the library's
//     device code is loaded, for as long as the process lives;
//   * all calls on a device share the one array, and it keeps whatever the
//     last call left in it: two calls whose GPU work overlaps (different
//     streams, or different host threads) race on it and give wrong results,
//     so serialise them.  Every scratch word a call reads is written earlier
//     in the same call (keys, values, digit histograms of every tile, all
//     ncells + 1 cell-table entries, the particle count), so nothing has to
//     be cleared between calls.
//   * the array's host-side name is only a stand-in for it; every call looks
//     the device address up with cudaGetSymbolAddress for the current device
//     and context, so the address stays right after a cudaDeviceReset or when
//     another context becomes current (nothing is cached);
//   * the call cannot be captured in a CUDA graph: it copies n from host
//     memory and ends by waiting for its stream (cudaStreamSynchronize);
//   * errors: the launches' configurations are valid by construction for
//     every accepted size, and the call reports the copies' return codes and
//     the stream's result; it neither reads nor clears errors that other
//     work left on the thread (no cudaGetLastError).
#include <cstdint>

#include "../../include/mps_capi.h"
#include "cellsort.cuh"

namespace {

using namespace mpsb;

constexpr uint32_t kMaxP = MPS_NOALLOC_MAX_PARTICLES;
constexpr uint32_t kMaxC = MPS_NOALLOC_MAX_CELLS;
constexpr uint32_t kMaxTiles = (kMaxP + SORT_TILE - 1) / SORT_TILE;

// word offsets of the regions inside the array (each 256-byte aligned)
constexpr size_t round64(size_t w) { return (w + 63) & ~size_t(63); }
constexpr size_t kKeys0 = 0;
constexpr size_t kVals0 = kKeys0 + round64(kMaxP);
constexpr size_t kKeys1 = kVals0 + round64(kMaxP);
constexpr size_t kVals1 = kKeys1 + round64(kMaxP);
constexpr size_t kHist = kVals1 + round64(kMaxP);
constexpr size_t kCells = kHist + round64((size_t)SORT_RADIX * kMaxTiles);
constexpr size_t kCount = kCells + round64((size_t)kMaxC + 1);
constexpr size_t kWords = kCount + 64;

static __device__ __align__(256) uint32_t g_cellsort_scratch[kWords];

// Device address of g_cellsort_scratch in the current device's context,
// looked up on every call (a cached address would go stale when the context
// that loaded the module is destroyed, e.g. by cudaDeviceReset).
mps_status scratch_for_current_device(uint32_t** out) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_cellsort_scratch) != cudaSuccess || !p) return MPS_ERR_CUDA;
    *out = static_cast<uint32_t*>(p);
    return MPS_OK;
}

}  // namespace

extern "C" mps_status mps_cell_sort_dev_noalloc(const float* pos4_dev, uint32_t n, const mps_grid* gg,
                                                uint32_t* perm_dev, uint32_t* cell_of_dev, uint32_t* start_dev,
                                                uint32_t* end_dev, uint32_t* n_in_grid_dev, void* stream) {
    if (!gg || (n && (!pos4_dev || !perm_dev || !cell_of_dev)) || !start_dev || !end_dev || !n_in_grid_dev)
        return MPS_ERR_INVALID;
    if (gg->ncells == 0) return MPS_ERR_INVALID;
    if (n > kMaxP || gg->ncells > kMaxC) return MPS_ERR_CAPACITY;
    uint32_t* base = nullptr;
    mps_status st0 = scratch_for_current_device(&base);
    if (st0 != MPS_OK) return st0;
    cudaStream_t st = (cudaStream_t)stream;
    Grid g;
    g.left = gg->left;
    g.back = gg->back;
    g.bottom = gg->bottom;
    g.cell_size = gg->cell_size;
    g.cdx = gg->cdx;
    g.cdy = gg->cdy;
    g.cdz = gg->cdz;
    g.sheet = gg->cdx * gg->cdy;
    g.ncells = gg->ncells;
    g.dim = gg->dim;
    g.base = 0;
    g.cell_yz = gg->cell_yz > 0.f ? gg->cell_yz : gg->cell_size;
    g.reach = 1;  // the sort reads only the cell edges
    SortScratch s;
    s.tiles = sort_tiles(n > 0 ? n : 1);
    s.keys[0] = base + kKeys0;
    s.vals[0] = base + kVals0;
    s.keys[1] = base + kKeys1;
    s.vals[1] = base + kVals1;
    s.hist = base + kHist;
    uint32_t* cs = base + kCells;
    uint32_t* n_dev = base + kCount;
    if (cudaMemcpyAsync(n_dev, &n, sizeof n, cudaMemcpyHostToDevice, st) != cudaSuccess) return MPS_ERR_CUDA;
    launch_cell_keys_plain((const float4*)pos4_dev, n, g, s.keys[0], s.vals[0], st);
    const int r = launch_radix_sort(s, n_dev, sort_passes(g.ncells), n, st);
    launch_cell_start_plain(s.keys[r], n, g, cs, n_in_grid_dev, st);
    bool copies_ok = true;
    if (n) {
        copies_ok &= cudaMemcpyAsync(perm_dev, s.vals[r], n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st) ==
                     cudaSuccess;
        copies_ok &= cudaMemcpyAsync(cell_of_dev, s.keys[r], n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st) ==
                     cudaSuccess;
    }
    launch_cell_end_from_start(cs, g.ncells, start_dev, end_dev, st);
    const cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess || !copies_ok) return MPS_ERR_CUDA;
    return MPS_OK;
}
