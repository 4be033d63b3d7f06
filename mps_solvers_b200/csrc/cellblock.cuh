// cellblock.cuh -- cell-block staging for the fast-arithmetic stencil stages.
//
// The reference's linked cells have the edge of the largest stencil radius
// (max(r0, rlap) = 4 l0), so walking a particle's 27 cells visits ~1,000
// candidates for the ~32 neighbours within r0 and ~1,400 for the ~250 within
// rlap; the stages are bound by issuing those candidate tests.  Here one
// thread block takes one coarse cell c:
//
//  1. it stages the particles of the 3 x 3 x 3 coarse cells around c (the
//     only cells a particle of c can reach) in shared memory: positions and
//     particle indices;
//  2. it sorts them by sub-cell of edge cell/3 (a 9 x 9 x 9 grid over the
//     block) with a stable counting sort: per-warp stable ranks from
//     __match_any_sync over the staging order, per-warp counts combined in
//     warp order, so the sorted order -- and every sum over it -- is the same
//     on every run;
//  3. each target particle of c (half a warp each) walks only the sub-cell
//     rows (dz, dy) its stencil radius can reach, each a contiguous range of
//     the sorted array, culled by the distance to the row.
//
// A particle's window [floor((x - re - m - x0) / h), floor((x + re + m - x0)
// / h)] (m a small margin) contains the sub-cell of every particle within re
// of it, computed with the same floor, so no neighbour is missed.  Sums are
// in sub-cell order, so these kernels serve the fast arithmetic only; the
// exact kernels keep the reference's candidate order.  A block whose 27
// cells hold more than CB_MAX particles stages nothing, and its targets walk
// the coarse cells from global memory instead (cb_fallback in the users).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "physics.cuh"

namespace mpsb {

constexpr int CB_THREADS = 128;
constexpr int CB_WARPS = CB_THREADS / 32;
constexpr uint32_t CB_MAX = 2048;   // staged particles of one block (1,728 lattice sites)
constexpr int CB_E = 9;             // sub-cells per block edge
constexpr int CB_NB = CB_E * CB_E * CB_E;

struct CbShared {
    float4 pos[CB_MAX];             // sorted by sub-cell
    uint32_t idx[CB_MAX];           // particle index of each sorted entry
    uint16_t key[CB_MAX];           // sub-cell of each staged particle (staging order)
    uint16_t rank[CB_MAX];          // its stable rank within its warp's segment
    uint16_t start[CB_NB + 1];      // first sorted entry of each sub-cell
    uint16_t wcnt[CB_WARPS][CB_NB]; // per-warp counts, then per-warp bases
    uint32_t pre[10];               // staging prefix over the 9 coarse rows
    uint32_t lo[9];                 // first particle of each coarse row
    uint32_t n;                     // staged particles (CB_MAX + 1: too many)
    float x0, y0, z0, h, inv_h;     // block origin and sub-cell edge
};

constexpr size_t CB_SMEM = sizeof(CbShared);

__device__ __forceinline__ int cb_sub(float v, float v0, float inv_h) {
    int s = (int)floorf((v - v0) * inv_h);
    return s < 0 ? 0 : (s > CB_E - 1 ? CB_E - 1 : s);
}

// Stage and sort the block of coarse cell c (all threads of the block).
// Returns false when it holds more than CB_MAX particles.
static __device__ __noinline__ bool cb_stage(CbShared& S, const Grid& g, const uint32_t* __restrict__ cs, uint32_t c,
                         const float4* __restrict__ pos) {
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t cz = c / g.sheet, rem = c - cz * g.sheet;
    const uint32_t cy = rem / g.cdx, cx = rem - cy * g.cdx;
    if (tid == 0) {
        // the 9 coarse rows (dz, dy) of cells cx-1 .. cx+1 inside the grid
        uint32_t tot = 0;
        const int x_lo = cx > 0 ? (int)cx - 1 : 0, x_hi = cx + 1 < g.cdx ? (int)cx + 1 : (int)cx;
        for (int r = 0; r < 9; r++) {
            const int dz = r / 3 - 1, dy = r % 3 - 1;
            const int zz = (int)cz + dz, yy = (int)cy + dy;
            uint32_t a = 0, b = 0;
            if (zz >= 0 && zz < (int)g.cdz && yy >= 0 && yy < (int)g.cdy) {
                const uint32_t base = (uint32_t)zz * g.sheet + (uint32_t)yy * g.cdx;
                a = __ldg(cs + base + x_lo);
                b = __ldg(cs + base + x_hi + 1);
            }
            S.lo[r] = a;
            S.pre[r] = tot;
            tot += b - a;
        }
        S.pre[9] = tot;
        S.n = tot <= CB_MAX ? tot : CB_MAX + 1;
        S.h = g.cell_size * (1.f / 3.f);
        S.inv_h = 3.f / g.cell_size;
        S.x0 = g.left + g.cell_size * (float)((int)cx - 1);
        S.y0 = g.back + g.cell_size * (float)((int)cy - 1);
        S.z0 = g.bottom + g.cell_size * (float)((int)cz - 1);
    }
    for (uint32_t b = tid; b < (uint32_t)(CB_WARPS * CB_NB); b += blockDim.x) (&S.wcnt[0][0])[b] = 0;
    __syncthreads();
    const uint32_t n = S.n;
    if (n > CB_MAX) return false;
    // keys and per-warp stable ranks: warp w ranks the staging segment
    // [w n / W, (w + 1) n / W) in order, 32 at a time
    const uint32_t s_lo = warp * n / CB_WARPS, s_hi = (warp + 1) * n / CB_WARPS;
    for (uint32_t k0 = s_lo; k0 < s_hi; k0 += 32) {
        const uint32_t k = k0 + lane;
        const bool ok = k < s_hi;
        uint32_t key = 0xffffu;
        if (ok) {
            int r = 0;
            while (r < 8 && S.pre[r + 1] <= k) r++;
            const uint32_t j = S.lo[r] + (k - S.pre[r]);
            const float4 p = __ldg(pos + j);
            key = (uint32_t)((cb_sub(p.z, S.z0, S.inv_h) * CB_E + cb_sub(p.y, S.y0, S.inv_h)) * CB_E +
                             cb_sub(p.x, S.x0, S.inv_h));
        }
        const uint32_t peers = __match_any_sync(0xffffffffu, key);
        uint32_t base = 0;
        if (ok) base = S.wcnt[warp][key];
        __syncwarp();
        if (ok) {
            S.key[k] = (uint16_t)key;
            S.rank[k] = (uint16_t)(base + __popc(peers & ((1u << lane) - 1u)));
            if ((peers & ((1u << lane) - 1u)) == 0) S.wcnt[warp][key] = (uint16_t)(base + __popc(peers));
        }
        __syncwarp();
    }
    __syncthreads();
    // per sub-cell: its total and the warps' bases in warp order
    for (uint32_t b = tid; b < (uint32_t)CB_NB; b += blockDim.x) {
        uint32_t t = 0;
#pragma unroll
        for (int w = 0; w < CB_WARPS; w++) {
            const uint32_t c_ = S.wcnt[w][b];
            S.wcnt[w][b] = (uint16_t)t;
            t += c_;
        }
        S.start[b] = (uint16_t)t;  // totals, scanned next
    }
    __syncthreads();
    if (warp == 0) {  // exclusive scan of the 729 totals, 23 a lane
        constexpr int PER = (CB_NB + 31) / 32;
        uint32_t v[PER];
        uint32_t sum = 0;
#pragma unroll
        for (int q = 0; q < PER; q++) {
            const uint32_t b = lane * PER + q;
            v[q] = b < (uint32_t)CB_NB ? S.start[b] : 0u;
            sum += v[q];
        }
        uint32_t inc = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= (uint32_t)o) inc += t;
        }
        uint32_t run = inc - sum;
#pragma unroll
        for (int q = 0; q < PER; q++) {
            const uint32_t b = lane * PER + q;
            if (b < (uint32_t)CB_NB) S.start[b] = (uint16_t)run;
            run += v[q];
        }
        if (lane == 31) S.start[CB_NB] = (uint16_t)inc;
    }
    __syncthreads();
    // scatter into sub-cell order
    for (uint32_t k = tid; k < n; k += blockDim.x) {
        uint32_t w = 0;
        while (w + 1 < (uint32_t)CB_WARPS && (w + 1) * n / CB_WARPS <= k) w++;
        int r = 0;
        while (r < 8 && S.pre[r + 1] <= k) r++;
        const uint32_t j = S.lo[r] + (k - S.pre[r]);
        const uint32_t key = S.key[k];
        const uint32_t slot = S.start[key] + S.wcnt[w][key] + S.rank[k];
        S.pos[slot] = __ldg(pos + j);
        S.idx[slot] = j;
    }
    __syncthreads();
    return true;
}

// The sub-cell rows a particle at p reaches within re: x, y and z ranges of
// sub-cells (inclusive), and (re + margin)^2.
struct CbWindow {
    int x0, x1, y0, y1, z0, z1;
    float re2;
};

__device__ __forceinline__ CbWindow cb_window(const CbShared& S, const float4& p, float re) {
    const float m = re + 1e-4f * S.h;
    CbWindow w;
    w.x0 = cb_sub(p.x - m, S.x0, S.inv_h);
    w.x1 = cb_sub(p.x + m, S.x0, S.inv_h);
    w.y0 = cb_sub(p.y - m, S.y0, S.inv_h);
    w.y1 = cb_sub(p.y + m, S.y0, S.inv_h);
    w.z0 = cb_sub(p.z - m, S.z0, S.inv_h);
    w.z1 = cb_sub(p.z + m, S.z0, S.inv_h);
    w.re2 = m * m;
    return w;
}

// Squared distance from v to the sub-cell slab s along one axis (0 inside).
__device__ __forceinline__ float cb_gap(float v, float v0, float h, int s) {
    const float a = v0 + h * (float)s, b = a + h;
    const float d = v < a ? a - v : (v > b ? v - b : 0.f);
    return d * d;
}

// Visit every staged candidate of the window's rows with half a warp (16
// lanes, hl = lane in the half): f(entry) for entries lo + hl, lo + hl + 16 ...
template <class F>
__device__ __forceinline__ void cb_walk(const CbShared& S, const float4& p, const CbWindow& w, uint32_t hl, F f) {
    for (int z = w.z0; z <= w.z1; z++) {
        const float gz = cb_gap(p.z, S.z0, S.h, z);
        if (gz >= w.re2) continue;
        for (int y = w.y0; y <= w.y1; y++) {
            const float gyz = gz + cb_gap(p.y, S.y0, S.h, y);
            if (gyz >= w.re2) continue;
            const int row = (z * CB_E + y) * CB_E;
            const uint32_t lo = S.start[row + w.x0], hi = S.start[row + w.x1 + 1];
            for (uint32_t e = lo + hl; e < hi; e += 16) f(e);
        }
    }
}

// The same walk with every lane of the half taking the same number of
// steps: f(entry, valid) with valid false past the end of a row, so that
// half-warp ballots inside f see all 16 lanes.
template <class F>
__device__ __forceinline__ void cb_walk_uniform(const CbShared& S, const float4& p, const CbWindow& w, uint32_t hl,
                                                F f) {
    for (int z = w.z0; z <= w.z1; z++) {
        const float gz = cb_gap(p.z, S.z0, S.h, z);
        if (gz >= w.re2) continue;
        for (int y = w.y0; y <= w.y1; y++) {
            const float gyz = gz + cb_gap(p.y, S.y0, S.h, y);
            if (gyz >= w.re2) continue;
            const int row = (z * CB_E + y) * CB_E;
            const uint32_t lo = S.start[row + w.x0], hi = S.start[row + w.x1 + 1];
            for (uint32_t e0 = lo; e0 < hi; e0 += 16) f(e0 + hl, e0 + hl < hi);
        }
    }
}

}  // namespace mpsb
