// cellsort.cu -- cell keys, stable radix sort by cell, cell tables.
//
// Replaces MPS_GPU::divideCell (MPS_CAL_expl_v1.0/MPS_GPU.cpp:248-331): the
// reference bins particles on the host with an atomic count, a serial prefix
// sum and a serial stable counting-sort rank.  Here the same stable order
// (particles grouped by cell, ascending previous index inside a cell) comes
// from an LSD radix sort on the cell id with the previous index as value.
#include "cellsort.cuh"

namespace mpsb {

// ---------------------------------------------------------------- keys
// In a batch each particle is binned in its own scene's grid and keyed by
// that grid's first global cell plus its cell there; outside its grid it
// takes the sentinel of all scenes' cells.
// key of particle i after the pending update
__device__ __forceinline__ uint32_t cell_key(const float4* __restrict__ pos, const float4* __restrict__ tmp, int apply,
                                             Grid g, Scalars* __restrict__ sc, const uint32_t* __restrict__ id,
                                             const BatchDev& batch, uint32_t i) {
    float4 p = pos[i];
    uint32_t s = 0;
    if (batch.n) {
        s = batch.sid_of_id[id[i]];
        g = batch.grid[s];
    }
    if (apply != APPLY_NONE && ptype(p) == T_FLUID) {
        const float dt = batch.n ? batch.dt[s] : sc->dt;
        float4 t = tmp[i];
        // x = x + dt * tmp, in float with one rounding per operation
        p.x = __fadd_rn(p.x, __fmul_rn(dt, t.x));
        p.y = __fadd_rn(p.y, __fmul_rn(dt, t.y));
        p.z = __fadd_rn(p.z, __fmul_rn(dt, t.z));
    }
    bool nan_flag = false;
    uint32_t k = cell_of_pos(g, p.x, p.y, p.z, &nan_flag);
    if (nan_flag) atomicOr(&sc->err, ERR_NAN);
    if (batch.n) k = k == g.ncells ? batch.ncells : g.base + k;
    return k;
}

// The keys fused with the first radix pass's upsweep: each block keys its
// tile of 2048 particles and counts their low digits (one launch less per
// rebuild).
__global__ void __launch_bounds__(SORT_THREADS) k_keys_upsweep(const float4* __restrict__ pos,
                                                               const float4* __restrict__ tmp, int apply, Grid g,
                                                               Scalars* __restrict__ sc, uint32_t* __restrict__ keys,
                                                               uint32_t* __restrict__ vals,
                                                               const uint32_t* __restrict__ id, BatchDev batch,
                                                               uint32_t* __restrict__ hist, uint32_t tiles) {
    __shared__ uint32_t h[SORT_RADIX];
    const uint32_t n = sc->np;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        sc->n_fluid = 0;  // the gather of this rebuild refills the particle lists
        sc->n_solid = 0;
    }
    for (int d = threadIdx.x; d < SORT_RADIX; d += SORT_THREADS) h[d] = 0;
    __syncthreads();
    const uint32_t base = blockIdx.x * SORT_TILE;
    if (base < n) {
#pragma unroll
        for (int k = 0; k < SORT_ITEMS; k++) {
            const uint32_t idx = base + k * SORT_THREADS + threadIdx.x;
            if (idx < n) {
                const uint32_t key = cell_key(pos, tmp, apply, g, sc, id, batch, idx);
                keys[idx] = key;
                vals[idx] = idx;
                atomicAdd(&h[key & 0xffu], 1u);
            }
        }
    }
    __syncthreads();
    for (int d = threadIdx.x; d < SORT_RADIX; d += SORT_THREADS) hist[d * tiles + blockIdx.x] = h[d];
}

__global__ void __launch_bounds__(256) k_cell_keys_plain(const float4* __restrict__ pos, uint32_t n, Grid g,
                                                         uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 p = pos[i];
    bool nan_flag = false;
    keys[i] = cell_of_pos(g, p.x, p.y, p.z, &nan_flag);
    vals[i] = i;
}

// ---------------------------------------------------------------- radix sort
// Upsweep: digit histogram of each tile, stored digit-major
// (hist[d * tiles + tile]) so that one exclusive scan over hist yields the
// global output offset of (digit, tile) for a stable LSD pass.
__global__ void __launch_bounds__(SORT_THREADS) k_radix_upsweep(const uint32_t* __restrict__ keys,
                                                                const uint32_t* __restrict__ n_dev, int shift,
                                                                uint32_t* __restrict__ hist, uint32_t tiles) {
    __shared__ uint32_t h[SORT_RADIX];
    const uint32_t n = *n_dev;
    for (int d = threadIdx.x; d < SORT_RADIX; d += SORT_THREADS) h[d] = 0;
    __syncthreads();
    const uint32_t base = blockIdx.x * SORT_TILE;
    if (base < n) {
#pragma unroll
        for (int k = 0; k < SORT_ITEMS; k++) {
            uint32_t idx = base + k * SORT_THREADS + threadIdx.x;
            if (idx < n) atomicAdd(&h[(keys[idx] >> shift) & 0xffu], 1u);
        }
    }
    __syncthreads();
    for (int d = threadIdx.x; d < SORT_RADIX; d += SORT_THREADS) hist[d * tiles + blockIdx.x] = h[d];
}

// Exclusive scan of `total` counters by one block: chunks of 16384 entries,
// each thread loading 16 consecutive counters as four 16-byte vectors (the
// array starts 16-byte aligned), a block scan of the thread sums, and a
// running carry between chunks.
__global__ void __launch_bounds__(1024) k_scan_exclusive(uint32_t* __restrict__ a, uint32_t total) {
    __shared__ uint32_t warp_sums[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t carry = 0;
    for (uint32_t c0 = 0; c0 < total; c0 += 16384) {
        const uint32_t b0 = c0 + 16 * threadIdx.x;
        const bool full = b0 + 16 <= total;
        uint32_t v[16];
        if (full) {
            const uint4* p = reinterpret_cast<const uint4*>(a + b0);
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const uint4 t = p[u];
                v[4 * u] = t.x;
                v[4 * u + 1] = t.y;
                v[4 * u + 2] = t.z;
                v[4 * u + 3] = t.w;
            }
        } else {
#pragma unroll
            for (int u = 0; u < 16; u++) v[u] = (b0 + u < total) ? a[b0 + u] : 0u;
        }
        uint32_t s = 0;
#pragma unroll
        for (int u = 0; u < 16; u++) s += v[u];
        uint32_t x = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += t;
        }
        if (lane == 31) warp_sums[warp] = x;
        __syncthreads();
        if (warp == 0) {
            uint32_t w = warp_sums[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += t;
            }
            warp_sums[lane] = w;
        }
        __syncthreads();
        uint32_t run = carry + (x - s) + (warp > 0 ? warp_sums[warp - 1] : 0u);
        const uint32_t chunk_total = warp_sums[31];
#pragma unroll
        for (int u = 0; u < 16; u++) {
            const uint32_t e = run;
            run += v[u];
            v[u] = e;
        }
        if (full) {
            uint4* p = reinterpret_cast<uint4*>(a + b0);
#pragma unroll
            for (int u = 0; u < 4; u++) p[u] = make_uint4(v[4 * u], v[4 * u + 1], v[4 * u + 2], v[4 * u + 3]);
        } else {
#pragma unroll
            for (int u = 0; u < 16; u++)
                if (b0 + u < total) a[b0 + u] = v[u];
        }
        carry += chunk_total;
        __syncthreads();  // warp_sums is rewritten by the next chunk
    }
}

// Downsweep: stable rank of every key inside its tile and scatter.
// Warp w of the block owns keys [tile + 256w, tile + 256w + 256) and walks
// them 32 at a time in index order; __match_any_sync groups equal digits in a
// round, and the group's running count in warp_hist[w][digit] gives each key
// its rank among equal digits before it in the warp.  An exclusive scan over
// warps per digit then orders the warps, and the upsweep scan orders tiles.
__global__ void __launch_bounds__(SORT_THREADS) k_radix_downsweep(
    const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in, uint32_t* __restrict__ keys_out,
    uint32_t* __restrict__ vals_out, const uint32_t* __restrict__ hist, const uint32_t* __restrict__ n_dev, int shift,
    uint32_t tiles, int scanned) {
    constexpr int WARPS = SORT_THREADS / 32;
    static_assert(SORT_THREADS == SORT_RADIX, "one digit per thread");
    __shared__ uint32_t warp_hist[WARPS][SORT_RADIX];
    __shared__ uint32_t tile_off[SORT_RADIX];
    __shared__ uint32_t dsum[WARPS];
    const uint32_t n = *n_dev;
    const uint32_t base = blockIdx.x * SORT_TILE;
    if (base >= n) return;  // the whole block exits together
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = threadIdx.x; k < WARPS * SORT_RADIX; k += SORT_THREADS) (&warp_hist[0][0])[k] = 0;
    if (scanned) {
        for (int d = threadIdx.x; d < SORT_RADIX; d += SORT_THREADS) tile_off[d] = hist[d * tiles + blockIdx.x];
    } else {
        // the scan done here from the raw tile histograms (few tiles): the
        // output offset of (digit d, this tile) is the count of all smaller
        // digits plus the count of digit d in the earlier tiles
        const int d = threadIdx.x;
        const uint32_t* hd = hist + (size_t)d * tiles;
        uint32_t tot = 0, pre = 0;
#pragma unroll 8
        for (uint32_t t = 0; t < tiles; t++) {
            const uint32_t v = hd[t];
            tot += v;
            pre += t < blockIdx.x ? v : 0u;
        }
        uint32_t x = tot;  // inclusive scan of the digit totals: warps, then warp sums
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) dsum[warp] = x;
        __syncthreads();
        uint32_t before = 0;
        for (int w = 0; w < warp; w++) before += dsum[w];
        tile_off[d] = before + x - tot + pre;
    }
    __syncthreads();

    uint32_t key[SORT_ITEMS], val[SORT_ITEMS], rank[SORT_ITEMS];
    const uint32_t lt_mask = (1u << lane) - 1u;
#pragma unroll
    for (int r = 0; r < SORT_ITEMS; r++) {
        const uint32_t idx = base + warp * (32 * SORT_ITEMS) + r * 32 + lane;
        const bool valid = idx < n;
        key[r] = valid ? keys_in[idx] : 0u;
        val[r] = valid ? vals_in[idx] : 0u;
        const uint32_t d = valid ? ((key[r] >> shift) & 0xffu) : 0x100u;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const int leader = __ffs(peers) - 1;
        uint32_t prev = 0;
        if (lane == leader && valid) {
            prev = warp_hist[warp][d];
            warp_hist[warp][d] = prev + __popc(peers);
        }
        prev = __shfl_sync(0xffffffffu, prev, leader);
        rank[r] = prev + __popc(peers & lt_mask);
        __syncwarp();
    }
    __syncthreads();
    // exclusive scan across warps for each digit
    for (int d = threadIdx.x; d < SORT_RADIX; d += SORT_THREADS) {
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < WARPS; w++) {
            uint32_t t = warp_hist[w][d];
            warp_hist[w][d] = run;
            run += t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < SORT_ITEMS; r++) {
        const uint32_t idx = base + warp * (32 * SORT_ITEMS) + r * 32 + lane;
        if (idx < n) {
            const uint32_t d = (key[r] >> shift) & 0xffu;
            const uint32_t dst = tile_off[d] + warp_hist[warp][d] + rank[r];
            keys_out[dst] = key[r];
            vals_out[dst] = val[r];
        }
    }
}

// ---------------------------------------------------------------- merge rebuild
// keys after the pending update; the changed particles (key != the cell they
// were sorted into) appended to m.changed through one atomic per warp
__global__ void __launch_bounds__(256) k_merge_keys(const float4* __restrict__ pos, const float4* __restrict__ tmp,
                                                    int apply, Grid g, Scalars* __restrict__ sc,
                                                    const uint32_t* __restrict__ id, BatchDev batch,
                                                    const uint32_t* __restrict__ cell_old, MergeScratch m) {
    const uint32_t n = sc->np;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        sc->n_fluid = 0;  // the merge gather refills the particle lists
        sc->n_solid = 0;
    }
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t lane = threadIdx.x & 31;
    bool ch = false;
    if (i < n) {
        const uint32_t k = cell_key(pos, tmp, apply, g, sc, id, batch, i);
        m.newkey[i] = k;
        ch = k != cell_old[i];
    }
    const uint32_t bal = __ballot_sync(0xffffffffu, ch);
    uint32_t base = 0;
    if (lane == 0 && bal) base = atomicAdd(&m.count[0], __popc(bal));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (ch) m.changed[base + __popc(bal & ((1u << lane) - 1u))] = i;
}

// ascending bitonic sort of P (a power of two) entries of x in the block's
// memory (shared or global), all threads of the block taking part
template <class T>
__device__ __forceinline__ void block_bitonic(T* x, uint32_t P) {
    for (uint32_t k = 2; k <= P; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t t = threadIdx.x; t < P; t += blockDim.x) {
                const uint32_t l = t ^ j;
                if (l > t) {
                    const T u = x[t], v = x[l];
                    if (((t & k) == 0) == (u > v)) {
                        x[t] = v;
                        x[l] = u;
                    }
                }
            }
            __syncthreads();
        }
    }
}

// One block: the changed list in its two orders, padded to a power of two
// with entries greater than any real one.  Up to MERGE_SMEM_CAP entries in
// shared memory; more (a state set from the host that moved many particles
// across cells) in the scratch arrays themselves, sized for every particle.
__global__ void __launch_bounds__(MERGE_SORT_THREADS) k_merge_sort(MergeScratch m) {
    extern __shared__ uint64_t msh[];
    const uint32_t cnt = *(volatile uint32_t*)&m.count[0];
    __syncthreads();
    if (threadIdx.x == 0) {
        m.count[1] = cnt;
        m.count[0] = 0;  // empty for the next rebuild's keys kernel
    }
    if (cnt == 0) return;
    if (cnt <= MERGE_SORT_THREADS) {
        // few (the common case): every entry's rank is the count of smaller
        // ones (the entries are distinct: they hold distinct positions)
        uint64_t* ka = msh;
        uint32_t* kb = reinterpret_cast<uint32_t*>(msh + MERGE_SORT_THREADS);
        const uint32_t t = threadIdx.x;
        uint64_t va = 0;
        uint32_t vb = 0;
        if (t < cnt) {
            vb = m.changed[t];
            va = ((uint64_t)m.newkey[vb] << 32) | vb;
            ka[t] = va;
            kb[t] = vb;
        }
        __syncthreads();
        if (t < cnt) {
            uint32_t ra = 0, rb = 0;
            for (uint32_t u = 0; u < cnt; u++) {
                ra += ka[u] < va ? 1u : 0u;
                rb += kb[u] < vb ? 1u : 0u;
            }
            m.a[ra] = va;
            m.b[rb] = vb;
        }
        return;
    }
    uint32_t P = 1;
    while (P < cnt) P <<= 1;
    const bool in_smem = P <= MERGE_SMEM_CAP;  // else m.a and m.b hold a power of two >= cap entries
    uint64_t* ka = in_smem ? msh : m.a;
    uint32_t* kb = in_smem ? reinterpret_cast<uint32_t*>(msh + MERGE_SMEM_CAP) : m.b;
    for (uint32_t t = threadIdx.x; t < P; t += blockDim.x) {
        if (t < cnt) {
            const uint32_t q = m.changed[t];
            ka[t] = ((uint64_t)m.newkey[q] << 32) | q;
            kb[t] = q;
        } else {
            ka[t] = ~0ull;
            kb[t] = ~0u;
        }
    }
    __syncthreads();
    block_bitonic(ka, P);
    block_bitonic(kb, P);
    if (in_smem)
        for (uint32_t t = threadIdx.x; t < cnt; t += blockDim.x) {
            m.a[t] = ka[t];
            m.b[t] = kb[t];
        }
}

cudaError_t merge_sort_setup() {
    return cudaFuncSetAttribute(k_merge_sort, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(MERGE_SMEM_CAP * (sizeof(uint64_t) + sizeof(uint32_t))));
}

void launch_merge_keys_sort(const float4* pos, const float4* tmp, int apply, const Grid& g, Scalars* sc,
                            const uint32_t* id, const BatchDev& batch, const uint32_t* cell_old,
                            const MergeScratch& m, uint32_t cap, cudaStream_t st) {
    k_merge_keys<<<(cap + 255) / 256, 256, 0, st>>>(pos, tmp, apply, g, sc, id, batch, cell_old, m);
    k_merge_sort<<<1, MERGE_SORT_THREADS, MERGE_SMEM_CAP * (sizeof(uint64_t) + sizeof(uint32_t)), st>>>(m);
}

// ---------------------------------------------------------------- cell tables
// (cell_start_fill is in cellsort.cuh; the particle steps' rebuild fills the
// table in its gather kernel)
__global__ void __launch_bounds__(256) k_cell_start_plain(const uint32_t* __restrict__ keys, uint32_t n, Grid g,
                                                          uint32_t* __restrict__ cell_start,
                                                          uint32_t* __restrict__ n_in_grid) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > n) return;
    cell_start_fill(keys, n, g.ncells, p, cell_start);
    long long prev = p > 0 ? (long long)keys[p - 1] : -1ll;
    long long cur = p < n ? (long long)keys[p] : (long long)g.ncells;
    if (prev < (long long)g.ncells && cur >= (long long)g.ncells) *n_in_grid = p;
}

__global__ void k_start_end(const uint32_t* __restrict__ cs, uint32_t ncells, uint32_t* __restrict__ start,
                            uint32_t* __restrict__ end) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    start[c] = cs[c];
    end[c] = cs[c + 1];
}

// ---------------------------------------------------------------- launchers
static inline uint32_t blocks_for(uint32_t n, uint32_t t) { return (n + t - 1) / t; }


static int radix_passes(SortScratch& s, const uint32_t* n_dev, int passes, cudaStream_t st, bool first_counted) {
    int cur = 0;
    for (int p = 0; p < passes; p++) {
        const int shift = 8 * p;
        if (!(p == 0 && first_counted))
            k_radix_upsweep<<<s.tiles, SORT_THREADS, 0, st>>>(s.keys[cur], n_dev, shift, s.hist, s.tiles);
        // few tiles: each downsweep block scans the histograms itself (one
        // launch less per pass); many: one scan kernel
        const int scanned = s.tiles > SORT_FUSED_SCAN_TILES;
        if (scanned) k_scan_exclusive<<<1, 1024, 0, st>>>(s.hist, SORT_RADIX * s.tiles);
        k_radix_downsweep<<<s.tiles, SORT_THREADS, 0, st>>>(s.keys[cur], s.vals[cur], s.keys[cur ^ 1],
                                                             s.vals[cur ^ 1], s.hist, n_dev, shift, s.tiles, scanned);
        cur ^= 1;
    }
    return cur;
}

int launch_radix_sort(SortScratch& s, const uint32_t* n_dev, int passes, uint32_t cap, cudaStream_t st) {
    (void)cap;
    return radix_passes(s, n_dev, passes, st, false);
}

int launch_keys_and_sort(const float4* pos, const float4* tmp, int apply, const Grid& g, Scalars* sc,
                         const uint32_t* id, const BatchDev& batch, SortScratch& s, int passes, cudaStream_t st) {
    k_keys_upsweep<<<s.tiles, SORT_THREADS, 0, st>>>(pos, tmp, apply, g, sc, s.keys[0], s.vals[0], id, batch, s.hist,
                                                     s.tiles);
    return radix_passes(s, &sc->np, passes, st, true);
}

void launch_scan_exclusive(uint32_t* a, uint32_t total, cudaStream_t st) {
    k_scan_exclusive<<<1, 1024, 0, st>>>(a, total);
}


void launch_cell_keys_plain(const float4* pos, uint32_t n, const Grid& g, uint32_t* keys, uint32_t* vals,
                            cudaStream_t st) {
    if (n == 0) return;
    k_cell_keys_plain<<<blocks_for(n, 256), 256, 0, st>>>(pos, n, g, keys, vals);
}

void launch_cell_start_plain(const uint32_t* keys_sorted, uint32_t n, const Grid& g, uint32_t* cell_start,
                             uint32_t* n_in_grid, cudaStream_t st) {
    k_cell_start_plain<<<blocks_for(n + 1, 256), 256, 0, st>>>(keys_sorted, n, g, cell_start, n_in_grid);
}

void launch_cell_end_from_start(const uint32_t* cell_start, uint32_t ncells, uint32_t* start_out, uint32_t* end_out,
                                cudaStream_t st) {
    if (ncells == 0) return;
    k_start_end<<<blocks_for(ncells, 256), 256, 0, st>>>(cell_start, ncells, start_out, end_out);
}

}  // namespace mpsb
