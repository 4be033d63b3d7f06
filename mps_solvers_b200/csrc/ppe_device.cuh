// ppe_device.cuh -- device helpers shared by the persistent PPE solvers:
// warp sums, the grid-wide reduction fused with a bounded grid barrier, and
// the L2-policy loads of the stored matrix.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "ppe.cuh"

namespace mpsb {

// ---------------------------------------------------------------- helpers
__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;  // every lane's value is used only from lane 0
}
__device__ __forceinline__ float warp_sum_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Grid-wide sum of K doubles fused with a grid barrier.  bar[0] counts
// arrivals and only grows during a launch (the assembly kernel empties it
// before every solve), so the e-th barrier of a launch completes when it
// reaches (e + 1) * gridDim.x and a block learns e from the count it saw
// before arriving.  Each block writes its fixed-order block sum into slot
// [e & 1][block] (two buffers: a block can write the slot of barrier e + 1
// only after every block has finished reading those of barrier e), arrives,
// waits for the count, and then adds all the slots itself in block order
// (lane-strided, then a fixed shuffle tree): the totals are identical in
// every block and on every run, and no block waits for another to publish
// them.  The wait is bounded: after 1 s (global timer) it sets
// ERR_DEVICE_TIMEOUT and returns false.
template <int K>
__device__ bool grid_reduce(const double (&v)[K], double* part, double* /*result*/, unsigned* bar, Scalars* sc,
                            double (&out)[K]) {
    __shared__ double sm[K][32];
    __shared__ double tot_s[K];
    __shared__ unsigned ep_s;
    __shared__ int ok_s;
    const unsigned G = gridDim.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    unsigned seen = 0;
    if (threadIdx.x == 0)  // the barrier's index, loaded early so the block sum hides the latency
        asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(seen) : "l"(bar) : "memory");
#pragma unroll
    for (int k = 0; k < K; k++) {
        const double t = warp_sum_d(v[k]);
        if (lane == 0) sm[k][warp] = t;
    }
    __syncthreads();
    if (warp == 0) {
        double t[K];
#pragma unroll
        for (int k = 0; k < K; k++) t[k] = warp_sum_d(lane < nw ? sm[k][lane] : 0.0);
        if (lane == 0) {
            const unsigned e = seen / G;
            double* slot = part + ((size_t)(e & 1u) * G + blockIdx.x) * PPE_PARTS;
#pragma unroll
            for (int k = 0; k < K; k++) slot[k] = t[k];
            __threadfence();  // this block's writes (slot and vectors) before the arrival
            atomicAdd(bar, 1u);
            const unsigned target = (e + 1) * G;
            int ok = 1;
            unsigned cur;
            uint64_t t0;
            const unsigned long long budget = wait_budget_ns(sc);
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
            for (;;) {
                asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(cur) : "l"(bar) : "memory");
                if ((int)(cur - target) >= 0) break;
                uint64_t t1;
                asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t1));
                if (t1 - t0 > budget) {
                    atomicOr(&sc->err, ERR_DEVICE_TIMEOUT);
                    ok = 0;
                    break;
                }
            }
            __threadfence();
            ep_s = e;
            ok_s = ok;
        }
    }
    __syncthreads();
    if (warp == 0) {
        const double* buf = part + (size_t)(ep_s & 1u) * G * PPE_PARTS;
#pragma unroll
        for (int k = 0; k < K; k++) {
            // up to 8 partials per lane loaded before adding (latency)
            double v8[8];
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const unsigned b = lane + 32u * u;
                v8[u] = b < G ? __ldcg(buf + b * PPE_PARTS + k) : 0.0;
            }
            double t = 0.0;
#pragma unroll
            for (int u = 0; u < 8; u++) t += v8[u];
            for (unsigned b = lane + 256u; b < G; b += 32) t += __ldcg(buf + b * PPE_PARTS + k);
            t = warp_sum_d(t);
            if (lane == 0) tot_s[k] = t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; k++) out[k] = tot_s[k];
    return ok_s != 0;
}


// L2 residency of the stored matrix.  Every CG iteration streams the whole
// matrix in the same order; once it is larger than L2 a plain LRU keeps none
// of it from one iteration to the next.  The entries before `keep` (the
// leading slices) are read as evict_last and the rest as evict_first, so the
// streamed tail displaces itself and the head stays in L2.  The matrix is
// read once per product, so it bypasses L1 (which keeps the gathered
// neighbour vectors instead).  keep = 0xFFFFFFFF reads everything with the
// default policy.
__device__ __forceinline__ uint64_t mat_policy(uint32_t base, uint32_t keep) {
    uint64_t p;
    if (keep == 0xFFFFFFFFu)
        asm("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(p));
    else if (base < keep)
        asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    else
        asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ uint4 ld_mat(const uint4* p, uint64_t pol) {
    uint4 v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
        : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
        : "l"(p), "l"(pol));
    return v;
}

__device__ __forceinline__ float4 ld_mat(const float4* p, uint64_t pol) {
    float4 v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
        : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
        : "l"(p), "l"(pol));
    return v;
}

// ---------------------------------------------------------------- learned S'
// The learned preconditioner S' = D^-1/2 S D^-1/2 (S the symmetric form of
// the network's factor) in sliced ELL with a thread per row: slices of 32
// consecutive row positions, width = the longest row of the slice, entry t
// of row position k at off[k / 32] + 32 t + k % 32.  Each entry is one
// 32-bit word: (column - c) in the upper 16 bits, the value in BF16 in the
// lower 16, where c is the row's own column (its compact position in the
// compact solver, its particle index in the particle-indexed solvers);
// padding is 0 (the row itself, value 0).  The diagonal is kept in FP32 by
// row position.
constexpr uint32_t SP_SLICE = 32;

// S' is read every iteration and is small next to the matrix: keep it in L2
__device__ __forceinline__ uint32_t sp_load(const uint32_t* p, uint64_t pol) {
    uint32_t v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
    return v;
}

// Row position k (own column c) of S' x, x_j given by a functor of the
// column.  Eight entries a round: their words first, then the eight x_j, so
// a row of ~25 entries costs four rounds of dependent loads.
template <class X>
__device__ __forceinline__ float sp_row_at(const uint32_t* __restrict__ off, const uint32_t* __restrict__ ent,
                                           const float* __restrict__ diag, uint32_t k, uint32_t c, X x) {
    const uint32_t s = k / SP_SLICE, lane = k % SP_SLICE;
    const uint32_t base = __ldg(off + s), W = (__ldg(off + s + 1) - base) / SP_SLICE;
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (uint32_t t0 = 0; t0 < W; t0 += 8) {
        uint32_t e[8];
#pragma unroll
        for (int u = 0; u < 8; u++)
            e[u] = t0 + u < W ? sp_load(ent + base + SP_SLICE * (size_t)(t0 + u) + lane, pol) : 0u;
        float xv[8];
#pragma unroll
        for (int u = 0; u < 8; u++) xv[u] = x((uint32_t)((int)c + ((int)e[u] >> 16)));
#pragma unroll
        for (int u = 0; u < 8; u++) acc[u] = fmaf(__uint_as_float(e[u] << 16), xv[u], acc[u]);
    }
    const float offd = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
    return fmaf(__ldg(diag + k), x(c), offd);
}

// A cooperative launch through the launch-attribute form, which stream
// capture records as a cooperative graph kernel node.
inline cudaError_t launch_cooperative_smem(const void* fn, int blocks, int threads, size_t smem, void** args,
                                           cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)blocks);
    cfg.blockDim = dim3((unsigned)threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelExC(&cfg, fn, args);
}

}  // namespace mpsb
