// ppe_compact.cu -- the PPE matrix in a compact 16-bit layout and the
// persistent PCG solve over it.
//
// Same system as ppe.cu (MPS_CPU::buildPoisson, MPS_CAL_v4.0/MPS_CPU.cpp:619-710,
// solved as MPS_CPU::DoCG's CG, :829-888, with diagonal scaling and FP64
// defect correction), stored for fewer bytes per CG iteration:
//
//  * unknowns are the R non-Dirichlet rows, numbered 0..R-1 in row-list
//    (ascending particle) order; every solver vector is indexed that way, so
//    the neighbour gathers touch a dense 8-byte-per-row vector;
//  * slices of 4 rows; a warp takes a slice with 8 lanes per row, lane
//    8 r + l holding entries 32 t + l, + 8, + 16 and + 24 of row r in chunk t
//    (rows padded to a multiple of 32 entries with weight 0), so the lanes
//    of a row gather 8 consecutive entries per instruction;
//  * a column is stored as 16 bits, column - 4 * slice + 32768 (the rows a
//    row couples to lie within a few cell layers of it in this numbering);
//    a column out of that range is stored as 65535 and its full value is
//    read from a side array with the same layout (escaped entries);
//  * weights FP32, beside the codes: 6 bytes per entry instead of 8.
//
// Per chunk a warp reads 256 contiguous bytes of codes and 512 of weights.
// The slices are dealt to warps round-robin; the same deal holds for the
// whole solve, so each warp keeps the last few chunks of its share in shared
// memory across all iterations, the matrix's head is read with an L2
// evict_last policy and the rest streams as evict_first.
#include <cstring>
#include <vector>

#include <cuda_bf16.h>

#include "cellsort.cuh"
#include "ppe.cuh"
#include "ppe_device.cuh"

namespace mpsb {

namespace {

inline uint32_t cblocks(uint32_t n, uint32_t t) { return (n + t - 1) / t; }

constexpr uint32_t C16_ROWS = 4;      // rows per slice
constexpr uint32_t C16_CHUNK = 128;   // entries per chunk (4 rows x 32)
constexpr uint32_t C16_ESC = 0xffffu; // escaped code
constexpr int C16_BIAS = 32768;

// Compact numbering of the rows, the rows' vectors in that numbering, and
// the chunk count of every slice (the longest of its 4 rows).  Thread k
// takes compact row k; 4 consecutive lanes form a slice.
__global__ void __launch_bounds__(256) k_c16_rows(const uint32_t* __restrict__ rowlist,
                                                  const uint32_t* __restrict__ nrows, const uint32_t* __restrict__ rlen,
                                                  const double* __restrict__ b64, const double* __restrict__ x64,
                                                  const double* __restrict__ diag64, const float* __restrict__ diag32,
                                                  const float* __restrict__ inv_diag, uint32_t* __restrict__ cpos,
                                                  double* __restrict__ cb64, double* __restrict__ cx64,
                                                  double* __restrict__ cdiag64, float* __restrict__ cdiag32,
                                                  float* __restrict__ cinv_diag, uint32_t* __restrict__ width,
                                                  uint32_t maxslices) {
    const uint32_t R = *nrows;
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t len = 0;
    if (k < R) {
        const uint32_t i = rowlist[k];
        cpos[i] = k;
        cb64[k] = b64[i];
        cx64[k] = x64[i];
        cdiag64[k] = diag64[i];
        cdiag32[k] = diag32[i];
        cinv_diag[k] = inv_diag[i];
        len = rlen[i];
    }
    len = max(len, __shfl_xor_sync(0xffffffffu, len, 1));
    len = max(len, __shfl_xor_sync(0xffffffffu, len, 2));
    const uint32_t s = k / C16_ROWS;
    if ((k & 3u) == 0 && s <= maxslices) width[s] = (len + 31u) / 32u;
}

// One warp per slice: the assembly's row-major columns (particle indices)
// and weights, recoded.  Lane L = 8 r + l writes, per chunk, its 4 codes as
// one 8-byte store and its 4 weights as one 16-byte store.
__global__ void __launch_bounds__(256) k_c16_pack(const uint32_t* __restrict__ cols_rm, const float* __restrict__ w_rm,
                                                  const uint32_t* __restrict__ rlen, const uint32_t* __restrict__ rowlist,
                                                  const uint32_t* __restrict__ nrows, const uint32_t* __restrict__ off,
                                                  const uint32_t* __restrict__ cpos, uint16_t* __restrict__ codes,
                                                  float* __restrict__ wts, uint32_t* __restrict__ side,
                                                  uint32_t* __restrict__ esc_count) {
    const uint32_t R = *nrows;
    const uint32_t slice = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31, r = lane >> 3, l = lane & 7;
    if (slice >= (R + C16_ROWS - 1) / C16_ROWS) return;
    const uint32_t g0 = off[slice];
    const uint32_t T = off[slice + 1] - g0;
    const uint32_t k = slice * C16_ROWS + r;
    const bool has = k < R;
    const uint32_t i = has ? rowlist[k] : 0u;
    const uint32_t len = has ? rlen[i] : 0u;
    const int base = (int)(slice * C16_ROWS) - C16_BIAS;
    const uint32_t pad = r + (uint32_t)C16_BIAS;  // the row itself, weight 0
    uint32_t nesc = 0;
    for (uint32_t t = 0; t < T; t++) {
        // lane 8 r + l holds entries l, l + 8, l + 16, l + 24 of the row's 32
        // in this chunk, so that one gather instruction of the solver reads
        // 8 consecutive entries of each row (neighbouring columns)
        const uint32_t e = 32u * t + l;
        uint32_t c[4] = {pad, pad, pad, pad};
        float w[4] = {0.f, 0.f, 0.f, 0.f};
        const size_t at = (size_t)(g0 + t) * C16_CHUNK + 4u * lane;
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const uint32_t eu = e + 8u * u;
            if (eu < len) {
                const uint32_t col = cpos[cols_rm[(size_t)i * PPE_W + eu]];
                const int code = (int)col - base;
                if (code >= 0 && code < (int)C16_ESC) {
                    c[u] = (uint32_t)code;
                } else {
                    c[u] = C16_ESC;
                    side[at + u] = col;
                    nesc++;
                }
                w[u] = w_rm[(size_t)i * PPE_W + eu];
            }
        }
        *reinterpret_cast<uint2*>(codes + at) = make_uint2(c[0] | (c[1] << 16), c[2] | (c[3] << 16));
        *reinterpret_cast<float4*>(wts + at) = make_float4(w[0], w[1], w[2], w[3]);
    }
    nesc = __reduce_add_sync(0xffffffffu, nesc);
    if (lane == 0 && nesc) atomicAdd(esc_count, nesc);
}

// p = max(x, 0) for the rows, 0 for Dirichlet particles (pressCorr,
// MPS_CAL_v4.0/MPS_CPU.cpp:734-743).
__global__ void __launch_bounds__(256) k_c16_finish(const double* __restrict__ cx64, const uint32_t* __restrict__ rlen,
                                                    const uint32_t* __restrict__ cpos, float* __restrict__ press,
                                                    const Scalars* __restrict__ sc) {
    const uint32_t n = sc->np;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float p = 0.f;
    if (rlen[i] != PPE_DIRICHLET) {
        p = (float)cx64[cpos[i]];
        if (p < 0.f) p = 0.f;
    }
    press[i] = p;
}

// Export: the stored entries of every row as particle indices, at
// row_start[i] (the particle's list) in stored order.
__global__ void __launch_bounds__(256) k_c16_export(const uint32_t* __restrict__ rlen,
                                                    const uint32_t* __restrict__ rowlist,
                                                    const uint32_t* __restrict__ nrows, const uint32_t* __restrict__ off,
                                                    const uint16_t* __restrict__ codes, const float* __restrict__ wts,
                                                    const uint32_t* __restrict__ side,
                                                    const uint32_t* __restrict__ row_start, uint32_t* __restrict__ cols,
                                                    float* __restrict__ out_w) {
    const uint32_t R = *nrows;
    const uint32_t slice = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31, r = lane >> 3, l = lane & 7;
    if (slice >= (R + C16_ROWS - 1) / C16_ROWS) return;
    const uint32_t k = slice * C16_ROWS + r;
    if (k >= R) return;
    const uint32_t g0 = off[slice], T = off[slice + 1] - g0;
    const uint32_t i = rowlist[k];
    const uint32_t len = rlen[i];
    const uint32_t o = row_start[i];
    const int base = (int)(slice * C16_ROWS) - C16_BIAS;
    for (uint32_t t = 0; t < T; t++)
        for (uint32_t u = 0; u < 4; u++) {
            const uint32_t e = 32u * t + l + 8u * u;  // the pack's order (k_c16_pack)
            if (e >= len) continue;
            const size_t at = (size_t)(g0 + t) * C16_CHUNK + 4u * lane + u;
            const uint32_t c = codes[at];
            const uint32_t col = c == C16_ESC ? side[at] : (uint32_t)(base + (int)c);
            cols[o + e] = rowlist[col];
            out_w[o + e] = wts[at];
        }
}

// ---------------------------------------------------------------- learned S'
// S' (its layout: ppe_device.cuh) of the current rows, from S kept by GEO
// index (learned.cuh): row position k holds its FP32 diagonal and its stored
// neighbours that are rows now.  A pair whose columns lie farther apart than
// 32,767 is left out from both its rows, which keeps S' symmetric and
// diagonally dominant (S is built dominant with a 1 % margin, more than BF16
// rounding of the entries takes away, so S' stays SPD).  PART selects the
// columns: particle indices (the particle-indexed solvers) or compact
// positions (the compact solver).
struct SpArgs {
    const uint32_t* rowlist;
    const uint32_t* nrows;
    const uint32_t* idv;       // GEO index of each particle
    const uint32_t* index_of_id;
    const uint32_t* rlen;
    const uint32_t* cpos;
    const double* diag64;      // particle-indexed diagonal of A
    const uint32_t* s_cnt;
    const uint32_t* s_col;
    const float* s_val;
    const float* s_diag;
    const Scalars* sc;
    uint32_t* off;             // widths (entries), then the scanned first entries
    uint32_t* ent;
    float* diag;
    uint32_t maxslices;
};

// The pack takes a thread per row (lane = row of the 32-row slice, so the
// packed words leave as coalesced 128-byte rows) and eight of its stored
// neighbours at a time, their loads issued together: the chain s_col ->
// index_of_id -> rlen, cpos, diag64 costs three dependent rounds per eight
// entries instead of per entry.
constexpr uint32_t SP_BATCH = 8;

// the batch [u0, u0 + 8) of the stored neighbours of a row with own column
// c: kept or not, the column offset and the neighbour's particle index
template <bool PART>
__device__ __forceinline__ void sp_batch(const SpArgs& A, uint32_t id, uint32_t n, uint32_t u0, uint32_t np,
                                         uint32_t c, bool (&ok)[SP_BATCH], int (&d)[SP_BATCH],
                                         uint32_t (&j)[SP_BATCH]) {
    uint32_t jd[SP_BATCH];
#pragma unroll
    for (uint32_t b = 0; b < SP_BATCH; b++)
        jd[b] = u0 + b < n ? __ldg(A.s_col + (size_t)id * LP_GW + u0 + b) : 0u;
#pragma unroll
    for (uint32_t b = 0; b < SP_BATCH; b++) j[b] = u0 + b < n ? __ldg(A.index_of_id + jd[b]) : np;
    uint32_t len[SP_BATCH], cp[SP_BATCH];
#pragma unroll
    for (uint32_t b = 0; b < SP_BATCH; b++) {
        const bool live = j[b] < np;
        len[b] = live ? __ldg(A.rlen + j[b]) : PPE_DIRICHLET;
        cp[b] = PART ? j[b] : (live ? __ldg(A.cpos + j[b]) : 0u);
    }
#pragma unroll
    for (uint32_t b = 0; b < SP_BATCH; b++) {
        d[b] = (int)cp[b] - (int)c;
        ok[b] = len[b] != PPE_DIRICHLET && d[b] >= -32767 && d[b] <= 32767;
    }
}

// Pass 1: off[s] = 32 x (the most stored entries of a row of slice s), every
// slice up to maxslices.  The stored count bounds the kept entries (the pack
// leaves out neighbours that are not rows now and far pairs, and pads the
// row with zeros), so this pass reads one count a row instead of following
// every entry to its row.
__global__ void __launch_bounds__(256) k_sp_width(SpArgs A) {
    const uint32_t R = *A.nrows;
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t s = k / SP_SLICE;
    uint32_t cnt = 0;
    if (k < R) cnt = __ldg(A.s_cnt + __ldg(A.idv + __ldg(A.rowlist + k)));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt = max(cnt, __shfl_xor_sync(0xffffffffu, cnt, o));
    if ((threadIdx.x & 31) == 0 && s <= A.maxslices) A.off[s] = cnt * SP_SLICE;
}

__device__ __forceinline__ uint32_t sp_bf16_bits(float v) {
    return (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(v));
}

// Pass 2 (after the scan of off): the kept entries of row k in stored order,
// then zeros up to the slice's width.
template <bool PART>
__global__ void __launch_bounds__(256) k_sp_pack(SpArgs A) {
    const uint32_t R = *A.nrows, np = A.sc->np;
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t s = k / SP_SLICE, lane = k % SP_SLICE;
    if (s >= (R + SP_SLICE - 1) / SP_SLICE) return;
    const uint32_t base = A.off[s], W = (A.off[s + 1] - base) / SP_SLICE;
    uint32_t t = 0;
    if (k < R) {
        const uint32_t i = __ldg(A.rowlist + k);
        const uint32_t id = __ldg(A.idv + i);
        const uint32_t n = __ldg(A.s_cnt + id);
        const float di = (float)(1.0 / sqrt(-__ldg(A.diag64 + i)));
        A.diag[k] = __ldg(A.s_diag + id) * (di * di);
        for (uint32_t u0 = 0; u0 < n; u0 += SP_BATCH) {
            bool ok[SP_BATCH];
            int d[SP_BATCH];
            uint32_t j[SP_BATCH];
            sp_batch<PART>(A, id, n, u0, np, PART ? i : k, ok, d, j);
            double dg[SP_BATCH];
            float sv[SP_BATCH];
#pragma unroll
            for (uint32_t b = 0; b < SP_BATCH; b++) {
                dg[b] = ok[b] ? __ldg(A.diag64 + j[b]) : -1.0;
                sv[b] = ok[b] ? __ldg(A.s_val + (size_t)id * LP_GW + u0 + b) : 0.f;
            }
#pragma unroll
            for (uint32_t b = 0; b < SP_BATCH; b++) {
                if (!ok[b]) continue;
                const float dj = (float)(1.0 / sqrt(-dg[b]));
                const float v = sv[b] * (di * dj);
                A.ent[base + SP_SLICE * t + lane] = ((uint32_t)(d[b] & 0xffff) << 16) | sp_bf16_bits(v);
                t++;
            }
        }
    }
    for (; t < W; t++) A.ent[base + SP_SLICE * t + lane] = 0u;
}

// ---------------------------------------------------------------- solve
struct C16Args {
    const uint32_t* nrows;
    const uint32_t* off;       // first chunk of every slice
    const uint16_t* codes;
    const float* wts;
    const uint32_t* side;
    const double* b64;
    const double* diag64;
    const float* diag32;
    const float* inv_diag;
    double* x64;
    float* r;
    float2* zp0;               // (z, p) per row: current and next
    float2* zp1;
    float* q;
    double* part;
    double* result;
    unsigned* bar;
    Scalars* sc;
    double tol, eta_min;
    uint32_t keep;             // chunks read as evict_last
    int max_iter, inner_cap, max_outer;
    int smem_chunks;           // chunks per warp held in shared memory
    // learned S' (LRN): slices of the same 4 rows, the second residual buffer
    const uint32_t* sp_off;
    const uint32_t* sp_ent;
    const float* sp_diag;
    float* r2;
};

// Row k of S' x on the compact rows (own column k).
template <class X>
__device__ __forceinline__ float sp_row(const C16Args& S, uint32_t k, X x) {
    return sp_row_at(S.sp_off, S.sp_ent, S.sp_diag, k, k, x);
}

// The four columns of a lane's chunk entries.
__device__ __forceinline__ void c16_cols(const uint2 cw, int base, const uint32_t* __restrict__ side, size_t at,
                                         uint32_t (&col)[4]) {
    col[0] = (uint32_t)(base + (int)(cw.x & 0xffffu));
    col[1] = (uint32_t)(base + (int)(cw.x >> 16));
    col[2] = (uint32_t)(base + (int)(cw.y & 0xffffu));
    col[3] = (uint32_t)(base + (int)(cw.y >> 16));
    if ((__vcmpeq2(cw.x, 0xffffffffu) | __vcmpeq2(cw.y, 0xffffffffu)) != 0u) {
        if ((cw.x & 0xffffu) == C16_ESC) col[0] = __ldg(side + at);
        if ((cw.x >> 16) == C16_ESC) col[1] = __ldg(side + at + 1);
        if ((cw.y & 0xffffu) == C16_ESC) col[2] = __ldg(side + at + 2);
        if ((cw.y >> 16) == C16_ESC) col[3] = __ldg(side + at + 3);
    }
}

__device__ __forceinline__ uint2 ld_codes(const uint2* p, uint64_t pol) {
    uint2 v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.u32 {%0, %1}, [%2], %3;"
        : "=r"(v.x), "=r"(v.y)
        : "l"(p), "l"(pol));
    return v;
}

__device__ __forceinline__ uint64_t c16_policy(uint32_t chunk, uint32_t keep) { return mat_policy(chunk, keep); }

// LRN: the learned preconditioner z = S' r instead of z = D^-1 r; S' is
// applied in the residual update (the neighbours' new residuals formed from
// r and q on the fly), so an iteration keeps two grid-wide reductions.
template <bool EX, bool LRN>
__global__ void __launch_bounds__(PPE_THREADS) k_ppe_solve_c16(C16Args S) {
    extern __shared__ __align__(16) unsigned char c16_sm[];
    const uint32_t R = *S.nrows;
    const uint32_t nsl = (R + C16_ROWS - 1) / C16_ROWS;
    const uint32_t lane = threadIdx.x & 31, rr = lane >> 3, l = lane & 7;
    const uint32_t wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    const uint32_t C = (uint32_t)S.smem_chunks;
    uint2* smc = reinterpret_cast<uint2*>(c16_sm) + (size_t)wib * C * 32;
    float4* smw = reinterpret_cast<float4*>(c16_sm + (size_t)wpb * C * 32 * sizeof(uint2)) + (size_t)wib * C * 32;
    const uint2* __restrict__ gcodes = reinterpret_cast<const uint2*>(S.codes);
    const float4* __restrict__ gw4 = reinterpret_cast<const float4*>(S.wts);

    // this warp's chunks, in the order it visits them; the last C of them
    // stay in shared memory for the whole solve
    uint32_t U = 0;
    for (uint32_t sl = gw; sl < nsl; sl += nw) U += __ldg(S.off + sl + 1) - __ldg(S.off + sl);
    const uint32_t u0 = U > C ? U - C : 0u;
    {
        uint32_t u = 0;
        for (uint32_t sl = gw; sl < nsl; sl += nw) {
            const uint32_t g0 = __ldg(S.off + sl), T = __ldg(S.off + sl + 1) - g0;
            for (uint32_t t = (u0 > u ? min(T, u0 - u) : 0u); t < T; t++) {
                const size_t g = (size_t)(g0 + t) * 32 + lane;
                smc[(u + t - u0) * 32 + lane] = __ldg(gcodes + g);
                smw[(u + t - u0) * 32 + lane] = __ldg(gw4 + g);
            }
            u += T;
        }
    }
    __syncwarp();

    int total = 0, outers = 0;
    double relres = 0.0;
    bool converged = false;
    float2* zc = S.zp0;
    float2* zn = S.zp1;
    float* rc = S.r;   // residual read by this iteration
    float* ra = S.r2;  // and the buffer its update writes (LRN)
    for (int outer = 0; outer < S.max_outer; outer++) {
        // ---- true residual r64 = b - A x64 (FP64); z = D^-1 r, p = 0
        double acc[3] = {0.0, 0.0, 0.0};
        uint32_t u = 0;
        for (uint32_t sl = gw; sl < nsl; sl += nw) {
            const uint32_t g0 = __ldg(S.off + sl), T = __ldg(S.off + sl + 1) - g0;
            const uint32_t ts = u0 > u ? min(T, u0 - u) : 0u;
            const int base = (int)(sl * C16_ROWS) - C16_BIAS;
            double s = 0.0;
            for (uint32_t t = 0; t < T; t++) {
                uint2 cw;
                float4 w;
                if (t < ts) {
                    const uint64_t pol = c16_policy(g0 + t, S.keep);
                    cw = ld_codes(gcodes + (size_t)(g0 + t) * 32 + lane, pol);
                    w = ld_mat(gw4 + (size_t)(g0 + t) * 32 + lane, pol);
                } else {
                    cw = smc[(u + t - u0) * 32 + lane];
                    w = smw[(u + t - u0) * 32 + lane];
                }
                uint32_t col[4];
                c16_cols(cw, base, S.side, (size_t)(g0 + t) * C16_CHUNK + 4u * lane, col);
                s += (double)w.x * S.x64[col[0]] + (double)w.y * S.x64[col[1]] + (double)w.z * S.x64[col[2]] +
                     (double)w.w * S.x64[col[3]];
            }
            u += T;
            s += __shfl_xor_sync(0xffffffffu, s, 1);
            s += __shfl_xor_sync(0xffffffffu, s, 2);
            s += __shfl_xor_sync(0xffffffffu, s, 4);
            const uint32_t k = sl * C16_ROWS + rr;
            if (l == 0 && k < R) {
                const double bi = S.b64[k];
                const double ri = bi - (S.diag64[k] * S.x64[k] + s);
                const float rf = (float)ri;
                rc[k] = rf;
                if (!LRN) {
                    const float zf = rf * S.inv_diag[k];
                    zc[k] = make_float2(zf, 0.f);
                    acc[2] += (double)rf * (double)zf;
                }
                acc[0] += ri * ri;
                acc[1] += bi * bi;
            }
        }
        double tot[3];
        if (!grid_reduce<3>(acc, S.part, S.result, S.bar, S.sc, tot)) return;
        outers++;
        const double rr64 = tot[0], bb = tot[1];
        relres = bb > 0.0 ? sqrt(rr64 / bb) : 0.0;
        if (relres <= S.tol) {
            converged = true;
            break;
        }
        if (total >= S.max_iter) break;
        if (LRN) {
            // z = S' r of the new residual, r.z
            double rz0[1] = {0.0};
            for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < R; k += gridDim.x * blockDim.x) {
                const float* rr_ = rc;
                const float zs = sp_row(S, k, [rr_](uint32_t j) { return rr_[j]; });
                zc[k] = make_float2(zs, 0.f);
                rz0[0] += (double)rc[k] * (double)zs;
            }
            double trz[1];
            if (!grid_reduce<1>(rz0, S.part, S.result, S.bar, S.sc, trz)) return;
            tot[2] = trz[0];
        }
        double eta = 0.3 * S.tol / relres;
        if (eta < S.eta_min) eta = S.eta_min;
        if (eta > 0.5) eta = 0.5;
        const double stop = eta * eta * rr64;
        double rz = tot[2];
        float beta = 0.f;
        for (int it = 0; it < S.inner_cap && total < S.max_iter; it++) {
            // ---- q = A p_new with p_new = z + beta p (fused), p.q
            double pq[1] = {0.0};
            u = 0;
            for (uint32_t sl = gw; sl < nsl; sl += nw) {
                const uint32_t g0 = __ldg(S.off + sl), T = __ldg(S.off + sl + 1) - g0;
                const uint32_t ts = u0 > u ? min(T, u0 - u) : 0u;
                const int base = (int)(sl * C16_ROWS) - C16_BIAS;
                float s0 = 0.f, s1 = 0.f;
#pragma unroll 2
                for (uint32_t t = 0; t < ts; t++) {
                    const uint64_t pol = c16_policy(g0 + t, S.keep);
                    const uint2 cw = ld_codes(gcodes + (size_t)(g0 + t) * 32 + lane, pol);
                    const float4 w = ld_mat(gw4 + (size_t)(g0 + t) * 32 + lane, pol);
                    uint32_t col[4];
                    c16_cols(cw, base, S.side, (size_t)(g0 + t) * C16_CHUNK + 4u * lane, col);
                    const float2 a0 = zc[col[0]], a1 = zc[col[1]], a2 = zc[col[2]], a3 = zc[col[3]];
                    s0 = fmaf(w.x, fmaf(beta, a0.y, a0.x), s0);
                    s1 = fmaf(w.y, fmaf(beta, a1.y, a1.x), s1);
                    s0 = fmaf(w.z, fmaf(beta, a2.y, a2.x), s0);
                    s1 = fmaf(w.w, fmaf(beta, a3.y, a3.x), s1);
                }
#pragma unroll 2
                for (uint32_t t = ts; t < T; t++) {
                    const uint2 cw = smc[(u + t - u0) * 32 + lane];
                    const float4 w = smw[(u + t - u0) * 32 + lane];
                    uint32_t col[4];
                    c16_cols(cw, base, S.side, (size_t)(g0 + t) * C16_CHUNK + 4u * lane, col);
                    const float2 a0 = zc[col[0]], a1 = zc[col[1]], a2 = zc[col[2]], a3 = zc[col[3]];
                    s0 = fmaf(w.x, fmaf(beta, a0.y, a0.x), s0);
                    s1 = fmaf(w.y, fmaf(beta, a1.y, a1.x), s1);
                    s0 = fmaf(w.z, fmaf(beta, a2.y, a2.x), s0);
                    s1 = fmaf(w.w, fmaf(beta, a3.y, a3.x), s1);
                }
                u += T;
                float s = s0 + s1;
                s += __shfl_xor_sync(0xffffffffu, s, 1);
                s += __shfl_xor_sync(0xffffffffu, s, 2);
                s += __shfl_xor_sync(0xffffffffu, s, 4);
                const uint32_t k = sl * C16_ROWS + rr;
                if (l == 0 && k < R) {
                    const float2 o = zc[k];
                    const float pn = fmaf(beta, o.y, o.x);
                    const float qi = fmaf(S.diag32[k], pn, s);
                    zn[k].y = pn;
                    S.q[k] = qi;
                    pq[0] += (double)pn * (double)qi;
                }
            }
            double totp[1];
            if (!grid_reduce<1>(pq, S.part, S.result, S.bar, S.sc, totp)) return;
            const double alpha = rz / totp[0];
            const float alpha_f = (float)alpha;
            // ---- x64 += alpha p, r -= alpha q, z = M^-1 r, r.z, r.r
            double acc2[2] = {0.0, 0.0};
            if (LRN) {
                // z_k = sum_j S'_kj (r_j - alpha q_j), the new residual into
                // the other buffer (the neighbours read the old one)
                for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < R; k += gridDim.x * blockDim.x) {
                    const float* rr_ = rc;
                    const float* qq_ = S.q;
                    const float zs =
                        sp_row(S, k, [rr_, qq_, alpha_f](uint32_t j) { return fmaf(-alpha_f, qq_[j], rr_[j]); });
                    const float pn = zn[k].y;
                    S.x64[k] += alpha * (double)pn;
                    const float ri = fmaf(-alpha_f, S.q[k], rc[k]);
                    ra[k] = ri;
                    zn[k] = make_float2(zs, pn);
                    acc2[0] += (double)ri * (double)zs;
                    acc2[1] += (double)ri * (double)ri;
                }
            } else {
                for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < R; k += gridDim.x * blockDim.x) {
                    const float pn = zn[k].y;
                    S.x64[k] += alpha * (double)pn;
                    const float ri = fmaf(-alpha_f, S.q[k], rc[k]);
                    const float zi = ri * S.inv_diag[k];
                    rc[k] = ri;
                    zn[k] = make_float2(zi, pn);
                    acc2[0] += (double)ri * (double)zi;
                    acc2[1] += (double)ri * (double)ri;
                }
            }
            double tot2[2];
            if (!grid_reduce<2>(acc2, S.part, S.result, S.bar, S.sc, tot2)) return;
            if (LRN) {
                float* t_ = rc;
                rc = ra;
                ra = t_;
            }
            total++;
            beta = (float)(tot2[0] / rz);
            rz = tot2[0];
            float2* tt = zc;
            zc = zn;
            zn = tt;
            if (tot2[1] <= stop) break;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        S.sc->cg_iters = total;
        S.sc->cg_outer = outers;
        S.sc->cg_relres = relres;
        if (!converged) atomicOr(&S.sc->err, ERR_CG_NOT_CONVERGED);
    }
}

template <class T>
bool c16_alloc(T** p, size_t count) {
    return cudaMalloc((void**)p, (count ? count : 1) * sizeof(T)) == cudaSuccess;
}

size_t c16_smem_bytes(int threads, int chunks) {
    return (size_t)(threads / 32) * (size_t)chunks * 32 * (sizeof(uint2) + sizeof(float4));
}

}  // namespace

int ppe_c16_enable(PpeWork& w, std::string* err) {
    if (w.c16_ready) return MPS_OK;
    const size_t cap = w.cap;
    const size_t vec = cap + 8;  // the last slice's padding rows read up to 3 past R
    const size_t slices = (cap + C16_ROWS - 1) / C16_ROWS + 2;
    w.c16_cap_chunks = slices * ((PPE_W + 31) / 32);
    const size_t ent = w.c16_cap_chunks * C16_CHUNK;
    bool ok = true;
    ok &= c16_alloc(&w.cpos, cap);
    ok &= c16_alloc(&w.c16_width, slices + 2);
    ok &= c16_alloc(&w.c16_codes, ent);
    ok &= c16_alloc(&w.c16_w, ent);
    ok &= c16_alloc(&w.c16_side, ent);
    ok &= c16_alloc(&w.c16_esc, 1);
    ok &= c16_alloc(&w.cb64, vec);
    ok &= c16_alloc(&w.cx64, vec);
    ok &= c16_alloc(&w.cdiag64, vec);
    ok &= c16_alloc(&w.cdiag32, vec);
    ok &= c16_alloc(&w.cinv_diag, vec);
    ok &= c16_alloc(&w.cr, vec);
    ok &= c16_alloc(&w.cq, vec);
    ok &= c16_alloc(&w.czp[0], vec);
    ok &= c16_alloc(&w.czp[1], vec);
    if (!ok) {
        ppe_c16_free(w);
        if (err) *err = "cudaMalloc failed for the compact PPE layout";
        return MPS_ERR_CUDA;
    }
    // padding rows beyond R read these: keep them finite
    cudaMemset(w.cx64, 0, vec * sizeof(double));
    cudaMemset(w.czp[0], 0, vec * sizeof(float2));
    cudaMemset(w.czp[1], 0, vec * sizeof(float2));
    const size_t most = c16_smem_bytes(PPE_THREADS, 8);
    if (cudaFuncSetAttribute(k_ppe_solve_c16<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)most) !=
            cudaSuccess ||
        cudaFuncSetAttribute(k_ppe_solve_c16<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)most) !=
            cudaSuccess ||
        cudaFuncSetAttribute(k_ppe_solve_c16<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)most) !=
            cudaSuccess ||
        cudaFuncSetAttribute(k_ppe_solve_c16<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)most) !=
            cudaSuccess) {
        ppe_c16_free(w);
        if (err) *err = "the compact PPE solver cannot have its shared memory";
        return MPS_ERR_CUDA;
    }
    w.c16_ready = true;
    return MPS_OK;
}

void ppe_c16_free(PpeWork& w) {
    void* ps[] = {w.cpos, w.c16_width, w.c16_codes, w.c16_w, w.c16_side, w.c16_esc, w.cb64, w.cx64, w.cdiag64,
                  w.cdiag32, w.cinv_diag, w.cr, w.cq, w.czp[0], w.czp[1], w.cr2};
    for (void* p : ps)
        if (p) cudaFree(p);
    w.cpos = w.c16_width = w.c16_esc = nullptr;
    w.c16_codes = nullptr;
    w.c16_w = nullptr;
    w.c16_side = nullptr;
    w.cb64 = w.cx64 = w.cdiag64 = nullptr;
    w.cdiag32 = w.cinv_diag = w.cr = w.cq = nullptr;
    w.czp[0] = w.czp[1] = nullptr;
    w.cr2 = nullptr;
    w.c16_ready = false;
    w.c16 = false;
    w.c16_learned = false;
}

int ppe_c16_enqueue_pack(PpeWork& w, const StageArgs& a, uint32_t cap, cudaStream_t st) {
    (void)a;
    const uint32_t maxslices = (cap + C16_ROWS - 1) / C16_ROWS;
    k_c16_rows<<<cblocks(C16_ROWS * (maxslices + 1), 256), 256, 0, st>>>(
        w.rowlist, w.nrows, w.rlen, w.b64, w.x64, w.diag64, w.diag32, w.inv_diag, w.cpos, w.cb64, w.cx64, w.cdiag64,
        w.cdiag32, w.cinv_diag, w.c16_width, maxslices);
    launch_scan_exclusive(w.c16_width, maxslices + 1, st);
    cudaMemsetAsync(w.c16_esc, 0, sizeof(uint32_t), st);
    k_c16_pack<<<cblocks(maxslices * 32u, 256), 256, 0, st>>>(w.cols, w.wrm, w.rlen, w.rowlist, w.nrows, w.c16_width,
                                                             w.cpos, w.c16_codes, w.c16_w, w.c16_side, w.c16_esc);
    return 3;
}

int ppe_c16_enqueue_solve(PpeWork& w, const StageArgs& a, const mps_options& opt, uint32_t cap, cudaStream_t st) {
    C16Args S;
    S.nrows = w.nrows;
    S.off = w.c16_width;
    S.codes = w.c16_codes;
    S.wts = w.c16_w;
    S.side = w.c16_side;
    S.b64 = w.cb64;
    S.diag64 = w.cdiag64;
    S.diag32 = w.cdiag32;
    S.inv_diag = w.cinv_diag;
    S.x64 = w.cx64;
    S.r = w.cr;
    S.zp0 = w.czp[0];
    S.zp1 = w.czp[1];
    S.q = w.cq;
    S.part = w.part;
    S.result = w.result;
    S.bar = w.bar;
    S.sc = a.sc;
    S.tol = opt.cg_tol;
    S.max_iter = opt.cg_max_iter;
    S.inner_cap = opt.cg_check_every > 0 ? opt.cg_check_every : 500;
    S.eta_min = pow(10.0, -(double)(opt.cg_inner_digits > 0 ? opt.cg_inner_digits : 4));
    S.max_outer = 40;
    // the matrix head kept in L2: the same byte budget as the 8-byte layout
    S.keep = w.l2_keep_entries == 0xFFFFFFFFu ? 0xFFFFFFFFu
                                               : (uint32_t)((size_t)w.l2_keep_entries * 8 / (C16_CHUNK * 6));
    // chunks per warp in shared memory (an SM holds 32 warps whichever the
    // block size, so the per-SM total is the same)
    int chunks = w.c16_smem_chunks;
    if (chunks < 0) chunks = 0;
    if (chunks > 8) chunks = 8;
    S.smem_chunks = chunks;
    const size_t smem = c16_smem_bytes(w.threads, chunks);
    S.sp_off = w.sp_off;
    S.sp_ent = w.sp_ent;
    S.sp_diag = w.sp_diag;
    S.r2 = w.cr2;
    void* args[] = {&S};
    const bool lrn = w.c16_learned;
    const void* fn = a.exact ? (lrn ? (const void*)k_ppe_solve_c16<true, true> : (const void*)k_ppe_solve_c16<true, false>)
                             : (lrn ? (const void*)k_ppe_solve_c16<false, true> : (const void*)k_ppe_solve_c16<false, false>);
    w.launch_err = launch_cooperative_smem(fn, w.blocks, w.threads, smem, args, st);
    if (!w.write_pressure) return 1;
    k_c16_finish<<<cblocks(cap, 256), 256, 0, st>>>(w.cx64, w.rlen, w.cpos, a.cur.press, a.sc);
    return 2;
}

int ppe_sp_enable(PpeWork& w, std::string* err) {
    if (lp_alloc_symmetric(w.lp) != MPS_OK) {
        if (err) *err = "cudaMalloc failed for the learned symmetric form";
        return MPS_ERR_CUDA;
    }
    if (w.sp_ent) return MPS_OK;
    const size_t slices = (w.cap + SP_SLICE - 1) / SP_SLICE + 2;
    w.sp_cap_chunks = slices * (LP_GW + 1);  // entries per lane position: 32-row slices of up to LP_GW + 1
    bool ok = c16_alloc(&w.sp_off, slices + 2);
    ok &= c16_alloc(&w.sp_ent, w.sp_cap_chunks * SP_SLICE);
    ok &= c16_alloc(&w.sp_diag, (size_t)w.cap + 8);
    ok &= c16_alloc(&w.rq[0], (size_t)w.cap + 8);
    ok &= c16_alloc(&w.rq[1], (size_t)w.cap + 8);
    if (!ok) {
        if (err) *err = "cudaMalloc failed for the learned preconditioner";
        return MPS_ERR_CUDA;
    }
    cudaMemset(w.rq[0], 0, ((size_t)w.cap + 8) * sizeof(float2));
    cudaMemset(w.rq[1], 0, ((size_t)w.cap + 8) * sizeof(float2));
    return MPS_OK;
}

int ppe_c16_learned_enable(PpeWork& w, std::string* err) {
    const int e = ppe_sp_enable(w, err);
    if (e != MPS_OK) return e;
    if (w.cr2) return MPS_OK;
    if (!c16_alloc(&w.cr2, (size_t)w.cap + 8)) {
        if (err) *err = "cudaMalloc failed for the learned compact preconditioner";
        return MPS_ERR_CUDA;
    }
    cudaMemset(w.cr2, 0, ((size_t)w.cap + 8) * sizeof(float));
    return MPS_OK;
}

int ppe_sp_enqueue_pack(PpeWork& w, const StageArgs& a, uint32_t cap, cudaStream_t st, bool by_particle) {
    SpArgs A;
    A.rowlist = w.rowlist;
    A.nrows = w.nrows;
    A.idv = a.cur.id;
    A.index_of_id = w.index_of_id;
    A.rlen = w.rlen;
    A.cpos = w.cpos;
    A.diag64 = w.diag64;
    A.s_cnt = w.lp.s_cnt;
    A.s_col = w.lp.s_col;
    A.s_val = w.lp.s_val;
    A.s_diag = w.lp.s_diag;
    A.sc = a.sc;
    A.off = w.sp_off;
    A.ent = w.sp_ent;
    A.diag = w.sp_diag;
    const uint32_t maxslices = (cap + SP_SLICE - 1) / SP_SLICE;
    A.maxslices = maxslices;
    const uint32_t wb = cblocks((maxslices + 1) * SP_SLICE, 256), pb = cblocks(maxslices * SP_SLICE, 256);
    k_sp_width<<<wb, 256, 0, st>>>(A);
    launch_scan_exclusive(w.sp_off, maxslices + 1, st);
    if (by_particle) k_sp_pack<true><<<pb, 256, 0, st>>>(A);
    else k_sp_pack<false><<<pb, 256, 0, st>>>(A);
    return 3;
}

int ppe_c16_export(const PpeWork& w, uint32_t np, const uint32_t* d_row_start, uint32_t* d_cols, float* d_w,
                   cudaStream_t st) {
    const uint32_t maxslices = (np + C16_ROWS - 1) / C16_ROWS;
    if (maxslices)
        k_c16_export<<<cblocks(maxslices * 32u, 256), 256, 0, st>>>(w.rlen, w.rowlist, w.nrows, w.c16_width,
                                                                   w.c16_codes, w.c16_w, w.c16_side, d_row_start,
                                                                   d_cols, d_w);
    return MPS_OK;
}

}  // namespace mpsb
