// learned.cu -- network, loss and training kernels of the learned PPE
// preconditioner (see learned.cuh for the model).
//
// Node arrays are indexed by particle and hold LP_H = 64 channels; every
// kernel iterates the ordered list of non-Dirichlet rows.  Edge kernels take
// one warp per row, lane l owning channels l and l+32.  Backward passes
// that would scatter to a neighbour instead gather over that neighbour's
// own stencil (the stencil is symmetric), so activation gradients are
// deterministic; parameter gradients are summed per block and added to the
// global gradient with atomics.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "cellsort.cuh"
#include "learned.cuh"
#include "ppe.cuh"

namespace mpsb {

static inline uint32_t blocks_for(uint32_t n, uint32_t t) { return (n + t - 1) / t; }

// ---------------------------------------------------------------- math
__device__ __forceinline__ float gelu_t(float x, float* dgelu) {
    const float k0 = 0.7978845608028654f, k1 = 0.044715f;
    const float u = k0 * (x + k1 * x * x * x);
    const float t = tanhf(u);
    if (dgelu) *dgelu = 0.5f * (1.f + t) + 0.5f * x * (1.f - t * t) * k0 * (1.f + 3.f * k1 * x * x);
    return 0.5f * x * (1.f + t);
}
__device__ __forceinline__ float softplus_f(float x) { return x > 20.f ? x : log1pf(expf(x)); }
__device__ __forceinline__ float sigmoid_f(float x) { return 1.f / (1.f + expf(-x)); }
__device__ __forceinline__ float wbf(const __nv_bfloat16* w, int k) { return __bfloat162float(w[k]); }

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// edge features of (i, j): dx, dy, dz, |r| over r0, w(r; r0), n_i / n0, [j wall]
struct Feat {
    float f[LP_F];
};
// r0 and 1/n0 of row i's scene
__device__ __forceinline__ float2 lp_consts(const LpSystem& S, uint32_t i) {
    if (S.phys) {
        const Phys& P = S.phys[__ldg(S.sid_of_id + __ldg(S.id + i))];
        return make_float2(P.rzero, P.one_over_nzero);
    }
    return make_float2(S.P.rzero, S.P.one_over_nzero);
}

__device__ __forceinline__ Feat edge_feat(const LpSystem& S, const float4& pi, float ni, uint32_t j, float2 k) {
    const float4 pj = __ldg(S.pos + j);
    const float inv = 1.f / k.x;
    const float dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
    const float r = sqrtf(dx * dx + dy * dy + dz * dz);
    Feat e;
    e.f[0] = dx * inv;
    e.f[1] = dy * inv;
    e.f[2] = dz * inv;
    e.f[3] = r * inv;
    e.f[4] = r > 0.f ? (k.x / r - 1.f) : 0.f;
    e.f[5] = ni * k.y;
    e.f[6] = ptype(pj) == T_WALL ? 1.f : 0.f;
    return e;
}

// ---------------------------------------------------------------- stencil
// One warp per non-Dirichlet row: its non-Dirichlet neighbours within r0 in
// ascending index (so the j < i entries come first), and D^-1/2.
__global__ void __launch_bounds__(256) k_lp_stencil(LpSystem S, uint32_t* __restrict__ scols,
                                                    uint32_t* __restrict__ scnt, uint32_t* __restrict__ nlow,
                                                    float* __restrict__ dinv, Scalars* __restrict__ sc) {
    const uint32_t R = *S.nrows;
    const uint32_t k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31, lt = (1u << lane) - 1u;
    if (k >= R) return;
    const uint32_t i = __ldg(S.rowlist + k);
    const float4 pi = __ldg(S.pos + i);
    Grid g = S.g;
    const uint32_t* cs = S.cell_start;
    uint32_t c = __ldg(S.cell + i);
    if (S.grids) {  // the row's scene grid; cells are numbered from its base
        g = S.grids[__ldg(S.sid_of_id + __ldg(S.id + i))];
        cs = S.cell_start + g.base;
        c -= g.base;
    }
    const float r0 = lp_consts(S, i).x;
    const float r02 = r0 * r0;
    uint32_t cnt = 0, low = 0;
    uint32_t* out = scols + (size_t)i * LP_GW;
    const CellNear nr = cell_near(g, c, pi.x, pi.y, pi.z, r0);
    auto visit = [&](uint32_t j, bool in) {
        {
            bool hit = false;
            if (in && j != i && __ldg(S.rlen + j) != PPE_DIRICHLET) {
                const float4 pj = __ldg(S.pos + j);
                const float dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
                hit = dx * dx + dy * dy + dz * dz < r02;
            }
            const uint32_t m = __ballot_sync(0xffffffffu, hit);
            if (hit) {
                const uint32_t t = cnt + __popc(m & lt);
                if (t < LP_GW) out[t] = j;
            }
            cnt += __popc(m);
            low += __popc(__ballot_sync(0xffffffffu, hit && j < i));
        }
    };
    if (g.reach > 1) walk_cells<true>(g, cs, c, nr, lane, visit);
    else walk_cells<false>(g, cs, c, nr, lane, visit);
    if (lane == 0) {
        if (cnt > LP_GW) {
            atomicOr(&sc->err, ERR_CAPACITY);
            cnt = LP_GW;
            if (low > cnt) low = cnt;
        }
        scnt[i] = cnt;
        nlow[i] = low;
        dinv[i] = (float)(1.0 / sqrt(-__ldg(S.diag64 + i)));
    }
}

// ---------------------------------------------------------------- forward
struct FwdArgs {
    LpSystem S;
    const uint32_t* scols;
    const uint32_t* scnt;
    const uint32_t* nlow;
    const __nv_bfloat16* w;
    float* a1;
    float* a2;
    const float* uh1;
    const float* ra;
    const float* rb;
    const float* h2;
    float* gval;
    float* gdiag;
    float* dgpre;
};

// the first (PASS == 1) or second message pass, mean-aggregated into a_out
template <int PASS>
__global__ void __launch_bounds__(256) k_lp_edge_fwd(FwdArgs A) {
    const LpSystem& S = A.S;
    const uint32_t R = *S.nrows;
    const uint32_t k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    if (k >= R) return;
    const uint32_t i = __ldg(S.rowlist + k);
    const int WE = PASS == 1 ? LP_W1E : LP_W2E;
    const int BB = PASS == 1 ? LP_B1 : LP_B2;
    float w0[LP_F], w1[LP_F];
#pragma unroll
    for (int f = 0; f < LP_F; f++) {
        w0[f] = wbf(A.w, WE + lane * LP_F + f);
        w1[f] = wbf(A.w, WE + (lane + 32) * LP_F + f);
    }
    const float b0 = wbf(A.w, BB + lane), b1 = wbf(A.w, BB + lane + 32);
    const float4 pi = __ldg(S.pos + i);
    const float2 kc = lp_consts(S, i);
    const float ni = __ldg(S.n + i);
    const uint32_t cnt = A.scnt[i];
    float acc0 = 0.f, acc1 = 0.f;
    for (uint32_t t = 0; t < cnt; t++) {
        const uint32_t j = A.scols[(size_t)i * LP_GW + t];
        const Feat e = edge_feat(S, pi, ni, j, kc);
        float s0 = b0, s1 = b1;
#pragma unroll
        for (int f = 0; f < LP_F; f++) {
            s0 = fmaf(w0[f], e.f[f], s0);
            s1 = fmaf(w1[f], e.f[f], s1);
        }
        if (PASS == 2) {
            s0 += A.uh1[(size_t)j * LP_H + lane];
            s1 += A.uh1[(size_t)j * LP_H + lane + 32];
        }
        acc0 += gelu_t(s0, nullptr);
        acc1 += gelu_t(s1, nullptr);
    }
    const float inv = cnt ? 1.f / (float)cnt : 0.f;
    float* a = PASS == 1 ? A.a1 : A.a2;
    a[(size_t)i * LP_H + lane] = acc0 * inv;
    a[(size_t)i * LP_H + lane + 32] = acc1 * inv;
}

// dense 64 -> 64 layer on every row: pre = W x + b (b optional), out =
// act(pre) + resid (act: 0 none, 1 GELU); 4 rows per 256-thread block.
__global__ void __launch_bounds__(256) k_lp_dense_fwd(const float* __restrict__ x, const __nv_bfloat16* __restrict__ w,
                                                      int woff, int boff, const float* __restrict__ resid,
                                                      float* __restrict__ pre_out, float* __restrict__ out, int act,
                                                      const uint32_t* __restrict__ rowlist,
                                                      const uint32_t* __restrict__ nrows) {
    __shared__ float W[LP_H][LP_H + 1];
    __shared__ float xs[4][LP_H];
    const uint32_t R = *nrows;
    for (int t = threadIdx.x; t < LP_H * LP_H; t += blockDim.x) W[t / LP_H][t % LP_H] = wbf(w, woff + t);
    const int r = threadIdx.x >> 6, o = threadIdx.x & 63;
    const float bias = boff >= 0 ? wbf(w, boff + o) : 0.f;
    for (uint32_t k0 = blockIdx.x * 4; k0 < R; k0 += gridDim.x * 4) {
        __syncthreads();
        const uint32_t k = k0 + r;
        const uint32_t i = k < R ? __ldg(rowlist + k) : 0u;
        if (k < R) xs[r][o] = x[(size_t)i * LP_H + o];
        __syncthreads();
        if (k < R) {
            float s = bias;
#pragma unroll 16
            for (int c = 0; c < LP_H; c++) s = fmaf(W[o][c], xs[r][c], s);
            if (pre_out) pre_out[(size_t)i * LP_H + o] = s;
            float v = act ? gelu_t(s, nullptr) : s;
            if (resid) v += resid[(size_t)i * LP_H + o];
            out[(size_t)i * LP_H + o] = v;
        }
    }
}

// readout: G_ij for the j < i entries, G_ii, and the pre-activation of G_ii
__global__ void __launch_bounds__(256) k_lp_readout_fwd(FwdArgs A) {
    const LpSystem& S = A.S;
    const uint32_t R = *S.nrows;
    const uint32_t k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    if (k >= R) return;
    const uint32_t i = __ldg(S.rowlist + k);
    float w0[LP_F], w1[LP_F];
#pragma unroll
    for (int f = 0; f < LP_F; f++) {
        w0[f] = wbf(A.w, LP_RE + lane * LP_F + f);
        w1[f] = wbf(A.w, LP_RE + (lane + 32) * LP_F + f);
    }
    const float ra0 = A.ra[(size_t)i * LP_H + lane] + wbf(A.w, LP_BR + lane);
    const float ra1 = A.ra[(size_t)i * LP_H + lane + 32] + wbf(A.w, LP_BR + lane + 32);
    const float om0 = wbf(A.w, LP_OM + lane), om1 = wbf(A.w, LP_OM + lane + 32);
    const float4 pi = __ldg(S.pos + i);
    const float2 kc = lp_consts(S, i);
    const float ni = __ldg(S.n + i);
    const uint32_t nl = A.nlow[i];
    for (uint32_t t = 0; t < nl; t++) {
        const uint32_t j = A.scols[(size_t)i * LP_GW + t];
        const Feat e = edge_feat(S, pi, ni, j, kc);
        float s0 = ra0 + A.rb[(size_t)j * LP_H + lane], s1 = ra1 + A.rb[(size_t)j * LP_H + lane + 32];
#pragma unroll
        for (int f = 0; f < LP_F; f++) {
            s0 = fmaf(w0[f], e.f[f], s0);
            s1 = fmaf(w1[f], e.f[f], s1);
        }
        const float g = warp_sum(om0 * gelu_t(s0, nullptr) + om1 * gelu_t(s1, nullptr));
        if (lane == 0) A.gval[(size_t)i * LP_GW + t] = g;
    }
    const float d = warp_sum(wbf(A.w, LP_DL + lane) * A.h2[(size_t)i * LP_H + lane] +
                             wbf(A.w, LP_DL + lane + 32) * A.h2[(size_t)i * LP_H + lane + 32]);
    if (lane == 0) {
        const float pre = d + wbf(A.w, LP_BD);
        A.dgpre[i] = pre;
        A.gdiag[i] = softplus_f(pre) + LP_GMIN;
    }
}

// the j > i entries of row i hold G_ji (found in row j's j < ... list)
__global__ void __launch_bounds__(256) k_lp_transpose(const uint32_t* __restrict__ scols, const uint32_t* __restrict__ scnt,
                                                      const uint32_t* __restrict__ nlow, float* __restrict__ v,
                                                      const uint32_t* __restrict__ rowlist,
                                                      const uint32_t* __restrict__ nrows) {
    const uint32_t R = *nrows;
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= R) return;
    const uint32_t i = rowlist[k];
    const uint32_t cnt = scnt[i];
    for (uint32_t t = nlow[i]; t < cnt; t++) {
        const uint32_t m = scols[(size_t)i * LP_GW + t];
        const uint32_t nm = nlow[m];
        float val = 0.f;
        // row m's lower entries are ascending: binary search for i
        uint32_t lo = 0, hi = nm;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (scols[(size_t)m * LP_GW + mid] < i) lo = mid + 1;
            else hi = mid;
        }
        if (lo < nm && scols[(size_t)m * LP_GW + lo] == i) val = v[(size_t)m * LP_GW + lo];
        v[(size_t)i * LP_GW + t] = val;
    }
}

// ---------------------------------------------------------------- sparse products
// y = G x (which = 0), y = G^T x (which = 1) on the non-Dirichlet rows
__global__ void __launch_bounds__(256) k_lp_gapply(const uint32_t* __restrict__ scols, const uint32_t* __restrict__ scnt,
                                                   const uint32_t* __restrict__ nlow, const float* __restrict__ gval,
                                                   const float* __restrict__ gdiag, const float* __restrict__ x,
                                                   float* __restrict__ y, int which,
                                                   const uint32_t* __restrict__ rowlist,
                                                   const uint32_t* __restrict__ nrows) {
    const uint32_t R = *nrows;
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= R) return;
    const uint32_t i = rowlist[k];
    const uint32_t t0 = which ? nlow[i] : 0u, t1 = which ? scnt[i] : nlow[i];
    float s = gdiag[i] * x[i];
    for (uint32_t t = t0; t < t1; t++) s = fmaf(gval[(size_t)i * LP_GW + t], x[scols[(size_t)i * LP_GW + t]], s);
    y[i] = s;
}

// y = Ahat x = x - D^-1/2 W D^-1/2 x (W: the rlap weights of the assembled A)
template <bool EX>
__global__ void __launch_bounds__(256) k_lp_ahat(LpSystem S, const float* __restrict__ dinv, const float* __restrict__ x,
                                                 float* __restrict__ y) {
    const uint32_t R = *S.nrows;
    const uint32_t k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    if (k >= R) return;
    const uint32_t i = __ldg(S.rowlist + k);
    const uint32_t len = __ldg(S.rlen + i);
    const float4 pi = __ldg(S.pos + i);
    float s = 0.f;
    for (uint32_t t = lane; t < len; t += 32) {
        const uint32_t j = __ldg(S.acols + (size_t)i * PPE_W + t);
        const float4 pj = __ldg(S.pos + j);
        const float dx = fsub<EX>(pj.x, pi.x), dy = fsub<EX>(pj.y, pi.y), dz = fsub<EX>(pj.z, pi.z);
        const float rr = dot3<EX>(dx, dy, dz, dx, dy, dz);
        const float w = rr < S.P.rlap_thr ? weight_rr<EX>(S.P.rlap, rr) : 0.f;
        s = fmaf(w * dinv[j], x[j], s);
    }
    s = warp_sum(s);
    if (lane == 0) y[i] = x[i] - dinv[i] * s;
}

// Rademacher probe from (seed, particle id); 0 off the rows
__global__ void __launch_bounds__(256) k_lp_probe(const uint32_t* __restrict__ ids, float* __restrict__ z, uint64_t seed,
                                                  const uint32_t* __restrict__ rowlist,
                                                  const uint32_t* __restrict__ nrows) {
    const uint32_t R = *nrows;
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= R) return;
    const uint32_t i = rowlist[k];
    uint64_t h = (seed << 32) + ids[i] + 0x9E3779B97F4A7C15ull;
    h = (h ^ (h >> 30)) * 0xBF58476D1CE4E5B9ull;
    h = (h ^ (h >> 27)) * 0x94D049BB133111EBull;
    h ^= h >> 31;
    z[i] = (h >> 63) ? 1.f : -1.f;
}

// Kaporin sums over the rows: T = v1 . v2 (= z^T G Ahat G^T z, the
// Hutchinson estimate of tr(G Ahat G^T)), sum log G_ii, and the row count
__global__ void __launch_bounds__(256) k_lp_kaporin(const float* __restrict__ v1, const float* __restrict__ v2,
                                                    const float* __restrict__ gdiag, double* __restrict__ sums,
                                                    const uint32_t* __restrict__ rowlist,
                                                    const uint32_t* __restrict__ nrows) {
    const uint32_t R = *nrows;
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    float t = 0.f, lg = 0.f;
    if (k < R) {
        const uint32_t i = rowlist[k];
        t = v1[i] * v2[i];
        lg = logf(gdiag[i]);
    }
    t = warp_sum(t);
    lg = warp_sum(lg);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(sums, (double)t);
        atomicAdd(sums + 1, (double)lg);
    }
}

// dL/dG for L = log(T / n) - (2 / n) sum log G_ii:
// dG_ij = (2 / T) z_i v2_j (j < i), dG_ii = (2 / T) z_i v2_i - 2 / (n G_ii)
__global__ void __launch_bounds__(256) k_lp_dg(const uint32_t* __restrict__ scols, const uint32_t* __restrict__ nlow,
                                               const float* __restrict__ v2, const float* __restrict__ z,
                                               const float* __restrict__ gdiag, const double* __restrict__ sums,
                                               float* __restrict__ dgval, float* __restrict__ dgdiag,
                                               const uint32_t* __restrict__ rowlist,
                                               const uint32_t* __restrict__ nrows) {
    const uint32_t R = *nrows;
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= R) return;
    const uint32_t i = rowlist[k];
    const float c = (float)(2.0 / sums[0]);
    const float cz = c * z[i];
    for (uint32_t t = 0; t < nlow[i]; t++) {
        const uint32_t j = scols[(size_t)i * LP_GW + t];
        dgval[(size_t)i * LP_GW + t] = cz * v2[j];
    }
    dgdiag[i] = cz * v2[i] - (float)(2.0 / (double)R) / gdiag[i];
}

// ---------------------------------------------------------------- backward
struct BwdArgs {
    LpSystem S;
    const uint32_t* scols;
    const uint32_t* scnt;
    const uint32_t* nlow;
    const __nv_bfloat16* w;
    const float *a1, *pre1, *h1, *uh1, *a2, *pre2, *h2, *ra, *rb, *dgpre;
    const float* dgval;   // dG, lower entries; upper entries hold dG of the transpose
    const float* dgdiag;
    float *dra, *drb, *dh2, *da;
    float* grad;
};

// readout, pass A (row i, its j < i entries): om, Re, br gradients, dra_i;
// G_ii: dl, bd gradients and dh2_i = dgpre_i * dl
__global__ void __launch_bounds__(256) k_lp_readout_bwd_a(BwdArgs A) {
    __shared__ float s_re[LP_H * LP_F];
    __shared__ float s_vec[3][LP_H];  // om, br, dl
    __shared__ float s_bd;
    for (int t = threadIdx.x; t < LP_H * LP_F; t += blockDim.x) s_re[t] = 0.f;
    for (int t = threadIdx.x; t < 3 * LP_H; t += blockDim.x) (&s_vec[0][0])[t] = 0.f;
    if (threadIdx.x == 0) s_bd = 0.f;
    __syncthreads();
    const LpSystem& S = A.S;
    const uint32_t R = *S.nrows;
    const uint32_t k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    float gre0[LP_F] = {0}, gre1[LP_F] = {0};
    float gom0 = 0.f, gom1 = 0.f, gbr0 = 0.f, gbr1 = 0.f, gdl0 = 0.f, gdl1 = 0.f, gbd = 0.f;
    if (k < R) {
        const uint32_t i = __ldg(S.rowlist + k);
        float w0[LP_F], w1[LP_F];
#pragma unroll
        for (int f = 0; f < LP_F; f++) {
            w0[f] = wbf(A.w, LP_RE + lane * LP_F + f);
            w1[f] = wbf(A.w, LP_RE + (lane + 32) * LP_F + f);
        }
        const float ra0 = A.ra[(size_t)i * LP_H + lane] + wbf(A.w, LP_BR + lane);
        const float ra1 = A.ra[(size_t)i * LP_H + lane + 32] + wbf(A.w, LP_BR + lane + 32);
        const float om0 = wbf(A.w, LP_OM + lane), om1 = wbf(A.w, LP_OM + lane + 32);
        const float4 pi = __ldg(S.pos + i);
        const float2 kc = lp_consts(S, i);
        const float ni = __ldg(S.n + i);
        float dra0 = 0.f, dra1 = 0.f;
        for (uint32_t t = 0; t < A.nlow[i]; t++) {
            const uint32_t j = A.scols[(size_t)i * LP_GW + t];
            const Feat e = edge_feat(S, pi, ni, j, kc);
            float s0 = ra0 + A.rb[(size_t)j * LP_H + lane], s1 = ra1 + A.rb[(size_t)j * LP_H + lane + 32];
#pragma unroll
            for (int f = 0; f < LP_F; f++) {
                s0 = fmaf(w0[f], e.f[f], s0);
                s1 = fmaf(w1[f], e.f[f], s1);
            }
            float d0, d1;
            const float g0 = gelu_t(s0, &d0), g1 = gelu_t(s1, &d1);
            const float dg = A.dgval[(size_t)i * LP_GW + t];
            gom0 += dg * g0;
            gom1 += dg * g1;
            const float dt0 = dg * om0 * d0, dt1 = dg * om1 * d1;
#pragma unroll
            for (int f = 0; f < LP_F; f++) {
                gre0[f] += dt0 * e.f[f];
                gre1[f] += dt1 * e.f[f];
            }
            gbr0 += dt0;
            gbr1 += dt1;
            dra0 += dt0;
            dra1 += dt1;
        }
        A.dra[(size_t)i * LP_H + lane] = dra0;
        A.dra[(size_t)i * LP_H + lane + 32] = dra1;
        // diagonal: G_ii = softplus(pre) + GMIN
        const float dpre = A.dgdiag[i] * sigmoid_f(A.dgpre[i]);
        const float h0 = A.h2[(size_t)i * LP_H + lane], h1v = A.h2[(size_t)i * LP_H + lane + 32];
        gdl0 = dpre * h0;
        gdl1 = dpre * h1v;
        gbd = lane == 0 ? dpre : 0.f;
        A.dh2[(size_t)i * LP_H + lane] = dpre * wbf(A.w, LP_DL + lane);
        A.dh2[(size_t)i * LP_H + lane + 32] = dpre * wbf(A.w, LP_DL + lane + 32);
    }
#pragma unroll
    for (int f = 0; f < LP_F; f++) {
        atomicAdd(&s_re[lane * LP_F + f], gre0[f]);
        atomicAdd(&s_re[(lane + 32) * LP_F + f], gre1[f]);
    }
    atomicAdd(&s_vec[0][lane], gom0);
    atomicAdd(&s_vec[0][lane + 32], gom1);
    atomicAdd(&s_vec[1][lane], gbr0);
    atomicAdd(&s_vec[1][lane + 32], gbr1);
    atomicAdd(&s_vec[2][lane], gdl0);
    atomicAdd(&s_vec[2][lane + 32], gdl1);
    if (gbd != 0.f) atomicAdd(&s_bd, gbd);
    __syncthreads();
    for (int t = threadIdx.x; t < LP_H * LP_F; t += blockDim.x) atomicAdd(A.grad + LP_RE + t, s_re[t]);
    for (int t = threadIdx.x; t < LP_H; t += blockDim.x) {
        atomicAdd(A.grad + LP_OM + t, s_vec[0][t]);
        atomicAdd(A.grad + LP_BR + t, s_vec[1][t]);
        atomicAdd(A.grad + LP_DL + t, s_vec[2][t]);
    }
    if (threadIdx.x == 0) atomicAdd(A.grad + LP_BD, s_bd);
}

// readout, pass B (row j, its j' > j entries = edges (i, j) with i > j):
// drb_j = sum_i dt_ij, recomputing dt_ij with the dG of (i, j)
__global__ void __launch_bounds__(256) k_lp_readout_bwd_b(BwdArgs A) {
    const LpSystem& S = A.S;
    const uint32_t R = *S.nrows;
    const uint32_t k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    if (k >= R) return;
    const uint32_t j = __ldg(S.rowlist + k);
    float w0[LP_F], w1[LP_F];
#pragma unroll
    for (int f = 0; f < LP_F; f++) {
        w0[f] = wbf(A.w, LP_RE + lane * LP_F + f);
        w1[f] = wbf(A.w, LP_RE + (lane + 32) * LP_F + f);
    }
    const float br0 = wbf(A.w, LP_BR + lane), br1 = wbf(A.w, LP_BR + lane + 32);
    const float om0 = wbf(A.w, LP_OM + lane), om1 = wbf(A.w, LP_OM + lane + 32);
    const float rbj0 = A.rb[(size_t)j * LP_H + lane], rbj1 = A.rb[(size_t)j * LP_H + lane + 32];
    float drb0 = 0.f, drb1 = 0.f;
    const uint32_t cnt = A.scnt[j];
    for (uint32_t t = A.nlow[j]; t < cnt; t++) {
        const uint32_t i = A.scols[(size_t)j * LP_GW + t];
        const float4 pi = __ldg(S.pos + i);
        const float2 kc = lp_consts(S, i);
        const Feat e = edge_feat(S, pi, __ldg(S.n + i), j, kc);
        float s0 = A.ra[(size_t)i * LP_H + lane] + br0 + rbj0;
        float s1 = A.ra[(size_t)i * LP_H + lane + 32] + br1 + rbj1;
#pragma unroll
        for (int f = 0; f < LP_F; f++) {
            s0 = fmaf(w0[f], e.f[f], s0);
            s1 = fmaf(w1[f], e.f[f], s1);
        }
        float d0, d1;
        gelu_t(s0, &d0);
        gelu_t(s1, &d1);
        const float dg = A.dgval[(size_t)j * LP_GW + t];  // transposed: dG of (i, j)
        drb0 += dg * om0 * d0;
        drb1 += dg * om1 * d1;
    }
    A.drb[(size_t)j * LP_H + lane] = drb0;
    A.drb[(size_t)j * LP_H + lane + 32] = drb1;
}

// dense backward on every row: dx (+)= W^T dy, dW += dy x^T, db += dy
__global__ void __launch_bounds__(256) k_lp_dense_bwd(const float* __restrict__ dy, const float* __restrict__ x,
                                                      const __nv_bfloat16* __restrict__ w, int woff, float* __restrict__ dx,
                                                      int accumulate, float* __restrict__ grad, int boff,
                                                      const uint32_t* __restrict__ rowlist,
                                                      const uint32_t* __restrict__ nrows) {
    __shared__ float W[LP_H][LP_H + 1];
    __shared__ float dW[LP_H][LP_H + 1];
    __shared__ float dys[4][LP_H], xs[4][LP_H];
    const uint32_t R = *nrows;
    for (int t = threadIdx.x; t < LP_H * LP_H; t += blockDim.x) {
        W[t / LP_H][t % LP_H] = wbf(w, woff + t);
        dW[t / LP_H][t % LP_H] = 0.f;
    }
    const int r = threadIdx.x >> 6, c = threadIdx.x & 63;
    float db = 0.f;
    for (uint32_t k0 = blockIdx.x * 4; k0 < R; k0 += gridDim.x * 4) {
        __syncthreads();
        const uint32_t k = k0 + r;
        const uint32_t i = k < R ? __ldg(rowlist + k) : 0u;
        dys[r][c] = k < R ? dy[(size_t)i * LP_H + c] : 0.f;
        xs[r][c] = k < R ? x[(size_t)i * LP_H + c] : 0.f;
        __syncthreads();
        if (k < R && dx) {
            float s = 0.f;
#pragma unroll 16
            for (int o = 0; o < LP_H; o++) s = fmaf(W[o][c], dys[r][o], s);
            if (accumulate) dx[(size_t)i * LP_H + c] += s;
            else dx[(size_t)i * LP_H + c] = s;
        }
        // dW[o][c'] for o = threadIdx.x / 4 .. : 256 threads x 16 entries
        const int o = threadIdx.x >> 2, c0 = (threadIdx.x & 3) * 16;
#pragma unroll
        for (int cc = 0; cc < 16; cc++) {
            float s = 0.f;
#pragma unroll
            for (int rr = 0; rr < 4; rr++) s = fmaf(dys[rr][o], xs[rr][c0 + cc], s);
            dW[o][c0 + cc] += s;
        }
        if (r == 0) {
#pragma unroll
            for (int rr = 0; rr < 4; rr++) db += dys[rr][c];
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < LP_H * LP_H; t += blockDim.x) atomicAdd(grad + woff + t, dW[t / LP_H][t % LP_H]);
    if (boff >= 0 && threadIdx.x < LP_H) atomicAdd(grad + boff + threadIdx.x, db);
}

// elementwise: out = dh * GELU'(pre)
__global__ void __launch_bounds__(256) k_lp_gelu_bwd(const float* __restrict__ dh, const float* __restrict__ pre,
                                                     float* __restrict__ out, const uint32_t* __restrict__ rowlist,
                                                     const uint32_t* __restrict__ nrows) {
    const uint32_t R = *nrows;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t k = t >> 6, c = t & 63;
    if (k >= R) return;
    const uint32_t i = rowlist[k];
    float d;
    gelu_t(pre[(size_t)i * LP_H + c], &d);
    out[(size_t)i * LP_H + c] = dh[(size_t)i * LP_H + c] * d;
}

__global__ void __launch_bounds__(256) k_lp_copy_rows(const float* __restrict__ src, float* __restrict__ dst,
                                                      const uint32_t* __restrict__ rowlist,
                                                      const uint32_t* __restrict__ nrows) {
    const uint32_t R = *nrows;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t k = t >> 6, c = t & 63;
    if (k >= R) return;
    const uint32_t i = rowlist[k];
    dst[(size_t)i * LP_H + c] = src[(size_t)i * LP_H + c];
}

// edge messages, pass A (row i): W{1,2}e and b{1,2} gradients from
// ds_ij = (da_i / cnt_i) * GELU'(s_ij)
template <int PASS>
__global__ void __launch_bounds__(256) k_lp_edge_bwd_a(BwdArgs A) {
    __shared__ float s_we[LP_H * LP_F];
    __shared__ float s_b[LP_H];
    for (int t = threadIdx.x; t < LP_H * LP_F; t += blockDim.x) s_we[t] = 0.f;
    for (int t = threadIdx.x; t < LP_H; t += blockDim.x) s_b[t] = 0.f;
    __syncthreads();
    const LpSystem& S = A.S;
    const uint32_t R = *S.nrows;
    const uint32_t k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    const int WE = PASS == 1 ? LP_W1E : LP_W2E;
    const int BB = PASS == 1 ? LP_B1 : LP_B2;
    float gw0[LP_F] = {0}, gw1[LP_F] = {0};
    float gb0 = 0.f, gb1 = 0.f;
    if (k < R) {
        const uint32_t i = __ldg(S.rowlist + k);
        float w0[LP_F], w1[LP_F];
#pragma unroll
        for (int f = 0; f < LP_F; f++) {
            w0[f] = wbf(A.w, WE + lane * LP_F + f);
            w1[f] = wbf(A.w, WE + (lane + 32) * LP_F + f);
        }
        const float b0 = wbf(A.w, BB + lane), b1 = wbf(A.w, BB + lane + 32);
        const float4 pi = __ldg(S.pos + i);
        const float2 kc = lp_consts(S, i);
        const float ni = __ldg(S.n + i);
        const uint32_t cnt = A.scnt[i];
        const float inv = cnt ? 1.f / (float)cnt : 0.f;
        const float da0 = A.da[(size_t)i * LP_H + lane] * inv, da1 = A.da[(size_t)i * LP_H + lane + 32] * inv;
        for (uint32_t t = 0; t < cnt; t++) {
            const uint32_t j = A.scols[(size_t)i * LP_GW + t];
            const Feat e = edge_feat(S, pi, ni, j, kc);
            float s0 = b0, s1 = b1;
#pragma unroll
            for (int f = 0; f < LP_F; f++) {
                s0 = fmaf(w0[f], e.f[f], s0);
                s1 = fmaf(w1[f], e.f[f], s1);
            }
            if (PASS == 2) {
                s0 += A.uh1[(size_t)j * LP_H + lane];
                s1 += A.uh1[(size_t)j * LP_H + lane + 32];
            }
            float d0, d1;
            gelu_t(s0, &d0);
            gelu_t(s1, &d1);
            const float ds0 = da0 * d0, ds1 = da1 * d1;
#pragma unroll
            for (int f = 0; f < LP_F; f++) {
                gw0[f] += ds0 * e.f[f];
                gw1[f] += ds1 * e.f[f];
            }
            gb0 += ds0;
            gb1 += ds1;
        }
    }
#pragma unroll
    for (int f = 0; f < LP_F; f++) {
        atomicAdd(&s_we[lane * LP_F + f], gw0[f]);
        atomicAdd(&s_we[(lane + 32) * LP_F + f], gw1[f]);
    }
    atomicAdd(&s_b[lane], gb0);
    atomicAdd(&s_b[lane + 32], gb1);
    __syncthreads();
    for (int t = threadIdx.x; t < LP_H * LP_F; t += blockDim.x) atomicAdd(A.grad + WE + t, s_we[t]);
    for (int t = threadIdx.x; t < LP_H; t += blockDim.x) atomicAdd(A.grad + BB + t, s_b[t]);
}

// second message pass, part B (row j): duh1_j = sum over the edges (i, j) of ds_ij
__global__ void __launch_bounds__(256) k_lp_edge2_bwd_b(BwdArgs A, float* __restrict__ duh1) {
    const LpSystem& S = A.S;
    const uint32_t R = *S.nrows;
    const uint32_t k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    if (k >= R) return;
    const uint32_t j = __ldg(S.rowlist + k);
    float w0[LP_F], w1[LP_F];
#pragma unroll
    for (int f = 0; f < LP_F; f++) {
        w0[f] = wbf(A.w, LP_W2E + lane * LP_F + f);
        w1[f] = wbf(A.w, LP_W2E + (lane + 32) * LP_F + f);
    }
    const float b0 = wbf(A.w, LP_B2 + lane) + A.uh1[(size_t)j * LP_H + lane];
    const float b1 = wbf(A.w, LP_B2 + lane + 32) + A.uh1[(size_t)j * LP_H + lane + 32];
    float acc0 = 0.f, acc1 = 0.f;
    const uint32_t cnt = A.scnt[j];
    for (uint32_t t = 0; t < cnt; t++) {
        const uint32_t i = A.scols[(size_t)j * LP_GW + t];
        const uint32_t ci = A.scnt[i];
        const float inv = ci ? 1.f / (float)ci : 0.f;
        const float4 pi = __ldg(S.pos + i);
        const float2 kc = lp_consts(S, i);
        const Feat e = edge_feat(S, pi, __ldg(S.n + i), j, kc);
        float s0 = b0, s1 = b1;
#pragma unroll
        for (int f = 0; f < LP_F; f++) {
            s0 = fmaf(w0[f], e.f[f], s0);
            s1 = fmaf(w1[f], e.f[f], s1);
        }
        float d0, d1;
        gelu_t(s0, &d0);
        gelu_t(s1, &d1);
        acc0 += A.da[(size_t)i * LP_H + lane] * inv * d0;
        acc1 += A.da[(size_t)i * LP_H + lane + 32] * inv * d1;
    }
    duh1[(size_t)j * LP_H + lane] = acc0;
    duh1[(size_t)j * LP_H + lane + 32] = acc1;
}

// ---------------------------------------------------------------- Adam
__global__ void k_lp_adam(float* __restrict__ w, __nv_bfloat16* __restrict__ w16, const float* __restrict__ g,
                          float* __restrict__ m, float* __restrict__ v, int n, float lr, float b1c, float b2c) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    float gk = g[k];
    if (!(gk == gk)) gk = 0.f;
    m[k] = b1 * m[k] + (1.f - b1) * gk;
    v[k] = b2 * v[k] + (1.f - b2) * gk * gk;
    const float mh = m[k] / b1c, vh = v[k] / b2c;
    w[k] -= lr * mh / (sqrtf(vh) + eps);
    w16[k] = __float2bfloat16(w[k]);
}

__global__ void k_lp_to_bf16(const float* __restrict__ w, __nv_bfloat16* __restrict__ w16, int n) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) w16[k] = __float2bfloat16(w[k]);
}

// ---------------------------------------------------------------- tensor-core dense layer
// The same 64 -> 64 layer on the fifth-generation tensor cores (inference):
// out = act(x W^T + b) + resid for a tile of 128 rows per step of a
// persistent CTA of 128 threads.  x is rounded to BF16 on its way into shared
// memory (W is BF16 already); the product accumulates in FP32 in tensor
// memory.  Operands use the no-swizzle K-major core-matrix layout (8 rows x
// 16 bytes per core matrix; element (m, k) at byte
// ((k / 8) * (M / 8) + m / 8) * 128 + (m % 8) * 16 + (k % 8) * 2), so one
// MMA of K = 16 reads two core-matrix columns: leading byte offset =
// M / 8 * 128 (the next 8 k), stride byte offset = 128 (the next 8 rows).
// One thread issues the 4 MMAs (K = 64) and commits them to an mbarrier;
// every thread waits on it (bounded), and each warp reads its 32 accumulator
// lanes with tcgen05.ld.
constexpr int TC_M = 128;
constexpr uint32_t TC_IDESC = (1u << 4)                  // accumulator F32
                              | (1u << 7) | (1u << 10)   // A, B BF16
                              | ((64u >> 3) << 17)       // N = 64
                              | ((128u >> 4) << 24);     // M = 128

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version of this architecture; no swizzle, base offset 0
    return d;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int k = 0; k < 16; k++) v[k] = __uint_as_float(r[k]);
}

// Shared memory of k_lp_dense_tc: A tile (BF16, K-major core matrices),
// W (BF16, same layout), and the FP32 accumulator staged for coalesced
// stores (row stride 68 floats: the row-per-thread writes and the
// half-warp-per-row reads are both free of bank conflicts).
constexpr uint32_t TC_SA = 0, TC_SB = TC_M * LP_H * 2, TC_SC = TC_SB + LP_H * LP_H * 2;
constexpr uint32_t TC_CST = LP_H + 4;
constexpr uint32_t TC_SMEM = TC_SC + TC_M * TC_CST * 4;

// wt: multiply by W^T instead of W (the backward pass's dx = W^T dy);
// accum: add the product to what out holds.
__global__ void __launch_bounds__(TC_M) k_lp_dense_tc(const float* __restrict__ x, const __nv_bfloat16* __restrict__ w,
                                                      int woff, int boff, const float* __restrict__ resid,
                                                      float* __restrict__ pre_out, float* __restrict__ out, int act,
                                                      const uint32_t* __restrict__ rowlist,
                                                      const uint32_t* __restrict__ nrows, uint32_t* __restrict__ err,
                                                      int wt, int accum) {
    extern __shared__ __align__(128) uint8_t smem[];
    uint8_t* sA = smem + TC_SA;
    uint8_t* sB = smem + TC_SB;
    float* sC = reinterpret_cast<float*>(smem + TC_SC);
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_slot;
    __shared__ int failed;
    const uint32_t R = *nrows;
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) failed = 0;
    // B (n, k) = W (n, k), or W (k, n) with wt, into the K-major layout,
    // N / 8 = 8 row groups
    for (uint32_t e = tid; e < LP_H * LP_H / 8; e += TC_M) {
        const uint32_t n = e / 8, kc = e % 8;  // row n, 8-element chunk kc
        uint4 v;
        if (!wt) {
            v = *reinterpret_cast<const uint4*>(w + woff + n * LP_H + kc * 8);
        } else {
            const unsigned short* wb = reinterpret_cast<const unsigned short*>(w + woff) + kc * 8 * LP_H + n;
            uint32_t u[4];
#pragma unroll
            for (int j = 0; j < 4; j++) u[j] = (uint32_t)wb[2 * j * LP_H] | ((uint32_t)wb[(2 * j + 1) * LP_H] << 16);
            v = make_uint4(u[0], u[1], u[2], u[3]);
        }
        *reinterpret_cast<uint4*>(sB + (kc * 8 + n / 8) * 128 + (n % 8) * 16) = v;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                     "r"(64));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&mbar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_slot;
    // epilogue columns of this lane (half-warp per row): 4 * (lane % 16) .. + 3
    const uint32_t ec = 4u * (lane & 15u);
    float4 bias = make_float4(0.f, 0.f, 0.f, 0.f);
    if (boff >= 0)
        bias = make_float4(__bfloat162float(w[boff + ec]), __bfloat162float(w[boff + ec + 1]),
                           __bfloat162float(w[boff + ec + 2]), __bfloat162float(w[boff + ec + 3]));
    uint32_t phase = 0;
    const uint32_t ntiles = (R + TC_M - 1) / TC_M;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        // A: warp w loads rows 32w .. 32w + 31 of the tile, 8 rows x 64 bytes
        // per instruction (lane: row r8 = lane / 4, float4 (lane % 4) of the
        // 64-byte column group g), converted to BF16 into the core matrices
        {
            const uint32_t r8 = lane >> 2, c4l = lane & 3u;
            uint32_t src[4];
#pragma unroll
            for (int rg = 0; rg < 4; rg++) {
                const uint32_t k = tile * TC_M + warp * 32 + rg * 8 + r8;
                src[rg] = k < R ? __ldg(rowlist + k) : 0xFFFFFFFFu;
            }
            float4 v[16];
#pragma unroll
            for (int rg = 0; rg < 4; rg++)
#pragma unroll
                for (int g = 0; g < 4; g++) {
                    const uint32_t i = src[rg];
                    v[rg * 4 + g] = i != 0xFFFFFFFFu
                                        ? __ldg(reinterpret_cast<const float4*>(x + (size_t)i * LP_H) + 4 * g + c4l)
                                        : make_float4(0.f, 0.f, 0.f, 0.f);
                }
#pragma unroll
            for (int rg = 0; rg < 4; rg++)
#pragma unroll
                for (int g = 0; g < 4; g++) {
                    const float4 a = v[rg * 4 + g];
                    const uint32_t c4 = 4 * g + c4l, m8 = warp * 4 + rg;  // float4 column, row group of 8
                    __nv_bfloat162 p0 = __floats2bfloat162_rn(a.x, a.y), p1 = __floats2bfloat162_rn(a.z, a.w);
                    uint2 u;
                    u.x = *reinterpret_cast<uint32_t*>(&p0);
                    u.y = *reinterpret_cast<uint32_t*>(&p1);
                    *reinterpret_cast<uint2*>(sA + ((c4 >> 1) * (TC_M / 8) + m8) * 128 + r8 * 16 + (c4 & 1u) * 8) = u;
                }
        }
        asm volatile("fence.proxy.async.shared::cta;");
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
            for (int kk = 0; kk < LP_H / 16; kk++) {
                const uint64_t da = umma_desc(smem_addr(sA) + kk * 2 * (TC_M / 8) * 128, (TC_M / 8) * 128, 128);
                const uint64_t db = umma_desc(smem_addr(sB) + kk * 2 * (LP_H / 8) * 128, (LP_H / 8) * 128, 128);
                const uint32_t acc = kk > 0 ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(TC_IDESC), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                smem_addr(&mbar)));
        }
        // bounded wait for the MMAs of this tile
        {
            uint32_t done = 0;
            for (uint32_t spin = 0; spin < (1u << 22) && !done; spin++) {
                asm volatile(
                    "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                    "selp.u32 %0, 1, 0, p;\n\t}\n"
                    : "=r"(done)
                    : "r"(smem_addr(&mbar)), "r"(phase));
                if (!done) __nanosleep(20);
            }
            if (!done) failed = 1;
        }
        phase ^= 1u;
        __syncthreads();
        if (failed) break;
        asm volatile("tcgen05.fence::after_thread_sync;");
        // TMEM lane = row of the tile: warp w reads rows 32w .. 32w + 31 and
        // stages them; the same warp then writes them out coalesced
        {
            float v[LP_H];
            const uint32_t lane_base = (warp * 32u) << 16;
#pragma unroll
            for (int c = 0; c < LP_H / 16; c++) tmem_ld16(tmem + lane_base + c * 16, v + 16 * c);
            asm volatile("tcgen05.wait::ld.sync.aligned;");
            float* row = sC + tid * TC_CST;
#pragma unroll
            for (int c = 0; c < LP_H / 4; c++)
                *reinterpret_cast<float4*>(row + 4 * c) = make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
        }
        __syncwarp();
#pragma unroll 4
        for (uint32_t it = 0; it < 16; it++) {
            const uint32_t m = warp * 32 + 2 * it + (lane >> 4);
            const uint32_t k = tile * TC_M + m;
            if (k < R) {
                const uint32_t i = __ldg(rowlist + k);
                const float4 a = *reinterpret_cast<const float4*>(sC + m * TC_CST + ec);
                const float4 sv = make_float4(a.x + bias.x, a.y + bias.y, a.z + bias.z, a.w + bias.w);
                const size_t o = (size_t)i * LP_H + ec;
                if (pre_out) *reinterpret_cast<float4*>(pre_out + o) = sv;
                float4 r = act ? make_float4(gelu_t(sv.x, nullptr), gelu_t(sv.y, nullptr), gelu_t(sv.z, nullptr),
                                             gelu_t(sv.w, nullptr))
                               : sv;
                if (resid) {
                    const float4 e = __ldg(reinterpret_cast<const float4*>(resid + o));
                    r.x += e.x;
                    r.y += e.y;
                    r.z += e.z;
                    r.w += e.w;
                }
                if (accum) {
                    const float4 e = *reinterpret_cast<const float4*>(out + o);
                    r.x += e.x;
                    r.y += e.y;
                    r.z += e.z;
                    r.w += e.w;
                }
                *reinterpret_cast<float4*>(out + o) = r;
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
    }
    if (tid == 0 && failed) atomicOr(err, ERR_DEVICE_TIMEOUT);
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(64));
    }
}

// ---------------------------------------------------------------- tensor-core weight gradient
// dW of a 64 -> 64 layer on the fifth-generation tensor cores (training):
// grad[woff + 64 o + c] += sum over the rows of dy(o) x(c), and
// grad[boff + o] += sum of dy(o) when boff >= 0.  The product is D = A B^T
// with the rows of the system as K, 128 of them a tile: A (M = 128) holds
// dy^T in its first 64 rows and zeros in the other 64 (written once), B
// (N = 64) holds x^T, both BF16 in the same no-swizzle K-major core-matrix
// layout as k_lp_dense_tc.  A persistent CTA accumulates all of its tiles in
// one 64-column FP32 accumulator in tensor memory (lane = o), then adds it
// to grad.  Staging: lane l of a warp takes features l and l + 32 of 8
// consecutive rows (eight coalesced 128-byte loads per operand and feature
// half), and writes each feature's 8 BF16 values as one 16-byte row of a
// core matrix; a warp's stores cover 512 contiguous bytes.  Eight warps a
// CTA, two k groups each, and two CTAs an SM keep enough loads in flight
// (with four warps and one CTA an SM the kernel ran at 16 % of DRAM peak).
constexpr uint32_t TW_K = 128, TW_THREADS = 256;
constexpr uint32_t TW_SA = 0, TW_SB = TC_M * TW_K * 2, TW_SMEM = TW_SB + LP_H * TW_K * 2;

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
    __nv_bfloat162 p = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&p);
}

__global__ void __launch_bounds__(TW_THREADS) k_lp_wgrad_tc(const float* __restrict__ dy, const float* __restrict__ x,
                                                      int woff, int boff, float* __restrict__ grad,
                                                      const uint32_t* __restrict__ rowlist,
                                                      const uint32_t* __restrict__ nrows, uint32_t* __restrict__ err) {
    extern __shared__ __align__(128) uint8_t smem[];
    uint8_t* sA = smem + TW_SA;
    uint8_t* sB = smem + TW_SB;
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_slot;
    __shared__ int failed;
    const uint32_t R = *nrows;
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) failed = 0;
    // rows 64 .. 127 of A are zero: (k group, row) units of 16 bytes
    for (uint32_t e = tid; e < (TW_K / 8) * 64; e += TW_THREADS) {
        const uint32_t kg = e / 64, m = 64 + e % 64;
        *reinterpret_cast<uint4*>(sA + (kg * (TC_M / 8) + m / 8) * 128 + (m % 8) * 16) = make_uint4(0u, 0u, 0u, 0u);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                     "r"(64));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&mbar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_slot;
    float db0 = 0.f, db1 = 0.f;  // bias gradient of features lane and lane + 32
    uint32_t phase = 0, ntile = 0;
    const uint32_t ntiles = (R + TW_K - 1) / TW_K;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        // warp w stages the k groups 2w and 2w + 1 of the tile
#pragma unroll 1
        for (uint32_t g = 0; g < 2; g++) {
            const uint32_t kg = warp * 2 + g;
            float a0[8], a1[8], b0[8], b1[8];
#pragma unroll
            for (int j = 0; j < 8; j++) {
                const uint32_t k = tile * TW_K + kg * 8 + j;
                if (k < R) {
                    const size_t o = (size_t)__ldg(rowlist + k) * LP_H + lane;
                    a0[j] = __ldg(dy + o);
                    a1[j] = __ldg(dy + o + 32);
                    b0[j] = __ldg(x + o);
                    b1[j] = __ldg(x + o + 32);
                } else {
                    a0[j] = a1[j] = b0[j] = b1[j] = 0.f;
                }
            }
#pragma unroll
            for (int j = 0; j < 8; j++) {
                db0 += a0[j];
                db1 += a1[j];
            }
            const uint32_t lo = (lane / 8) * 128 + (lane % 8) * 16, hi = lo + 4 * 128;  // features l, l + 32
            uint8_t* ra = sA + kg * (TC_M / 8) * 128;
            uint8_t* rb = sB + kg * (LP_H / 8) * 128;
            *reinterpret_cast<uint4*>(ra + lo) = make_uint4(pack_bf16x2(a0[0], a0[1]), pack_bf16x2(a0[2], a0[3]),
                                                            pack_bf16x2(a0[4], a0[5]), pack_bf16x2(a0[6], a0[7]));
            *reinterpret_cast<uint4*>(ra + hi) = make_uint4(pack_bf16x2(a1[0], a1[1]), pack_bf16x2(a1[2], a1[3]),
                                                            pack_bf16x2(a1[4], a1[5]), pack_bf16x2(a1[6], a1[7]));
            *reinterpret_cast<uint4*>(rb + lo) = make_uint4(pack_bf16x2(b0[0], b0[1]), pack_bf16x2(b0[2], b0[3]),
                                                            pack_bf16x2(b0[4], b0[5]), pack_bf16x2(b0[6], b0[7]));
            *reinterpret_cast<uint4*>(rb + hi) = make_uint4(pack_bf16x2(b1[0], b1[1]), pack_bf16x2(b1[2], b1[3]),
                                                            pack_bf16x2(b1[4], b1[5]), pack_bf16x2(b1[6], b1[7]));
        }
        asm volatile("fence.proxy.async.shared::cta;");
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
            for (int kk = 0; kk < (int)(TW_K / 16); kk++) {
                const uint64_t da = umma_desc(smem_addr(sA) + kk * 2 * (TC_M / 8) * 128, (TC_M / 8) * 128, 128);
                const uint64_t dbd = umma_desc(smem_addr(sB) + kk * 2 * (LP_H / 8) * 128, (LP_H / 8) * 128, 128);
                const uint32_t acc = (ntile > 0 || kk > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
                    "l"(da), "l"(dbd), "r"(TC_IDESC), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                smem_addr(&mbar)));
        }
        // bounded wait for this tile's MMAs (they read the staged operands)
        {
            uint32_t done = 0;
            for (uint32_t spin = 0; spin < (1u << 22) && !done; spin++) {
                asm volatile(
                    "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                    "selp.u32 %0, 1, 0, p;\n\t}\n"
                    : "=r"(done)
                    : "r"(smem_addr(&mbar)), "r"(phase));
                if (!done) __nanosleep(20);
            }
            if (!done) failed = 1;
        }
        phase ^= 1u;
        ntile++;
        __syncthreads();
        if (failed) break;
    }
    asm volatile("tcgen05.fence::after_thread_sync;");
    // accumulator rows 0 .. 63 (TMEM lanes of warps 0 and 1) through shared
    // memory (the A tile's space, stride 65 floats) to coalesced atomics
    float* sD = reinterpret_cast<float*>(sA);
    const bool have = ntile > 0 && !failed;
    if (have && warp < 2) {
        float v[LP_H];
        const uint32_t lane_base = (warp * 32u) << 16;
#pragma unroll
        for (int c = 0; c < LP_H / 16; c++) tmem_ld16(tmem + lane_base + c * 16, v + 16 * c);
        asm volatile("tcgen05.wait::ld.sync.aligned;");
#pragma unroll
        for (int c = 0; c < LP_H; c++) sD[tid * (LP_H + 1) + c] = v[c];
    }
    __syncthreads();
    if (have) {
        for (uint32_t t = tid; t < LP_H * LP_H; t += TW_THREADS)
            atomicAdd(grad + woff + t, sD[(t / LP_H) * (LP_H + 1) + t % LP_H]);
        if (boff >= 0) {
            atomicAdd(grad + boff + lane, db0);
            atomicAdd(grad + boff + lane + 32, db1);
        }
    }
    if (tid == 0 && failed) atomicOr(err, ERR_DEVICE_TIMEOUT);
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(64));
    }
}

// ---------------------------------------------------------------- host side
int lp_setup(LearnedWork& L, uint32_t cap, std::string* err) {
    L.cap = cap;
    bool ok = true;
    auto al = [&](void** p, size_t bytes) {
        if (cudaMalloc(p, bytes + 64) != cudaSuccess) { ok = false; return; }
        cudaMemset(*p, 0, bytes + 64);
    };
    const size_t N = cap, NH = (size_t)cap * LP_H, NG = (size_t)cap * LP_GW;
    al((void**)&L.w32, LP_NPARAM * 4);
    al((void**)&L.w16, LP_NPARAM * 2);
    al((void**)&L.grad, LP_NPARAM * 4);
    al((void**)&L.adam_m, LP_NPARAM * 4);
    al((void**)&L.adam_v, LP_NPARAM * 4);
    al((void**)&L.scols, NG * 4);
    al((void**)&L.scnt, N * 4);
    al((void**)&L.nlow, N * 4);
    al((void**)&L.gdiag, N * 4);
    al((void**)&L.gval, NG * 4);
    float** nodes[] = {&L.a1, &L.pre1, &L.h1, &L.uh1, &L.a2, &L.pre2, &L.h2, &L.ra, &L.rb};
    for (float** p : nodes) al((void**)p, NH * 4);
    al((void**)&L.dgpre, N * 4);
    al((void**)&L.dinv, N * 4);
    if (!ok) {
        *err = "cudaMalloc failed for the learned preconditioner";
        return MPS_ERR_CUDA;
    }
    std::vector<float> w(LP_NPARAM);
    lp_init_params(w.data(), 1234);
    lp_upload_params(L, w.data(), 0);
    cudaDeviceSynchronize();
    L.ready = true;
    return MPS_OK;
}

static int lp_setup_training(LearnedWork& L) {
    if (L.dh1) return MPS_OK;
    bool ok = true;
    auto al = [&](void** p, size_t bytes) {
        if (cudaMalloc(p, bytes + 64) != cudaSuccess) { ok = false; return; }
        cudaMemset(*p, 0, bytes + 64);
    };
    const size_t N = L.cap, NH = (size_t)L.cap * LP_H, NG = (size_t)L.cap * LP_GW;
    float** nodes[] = {&L.dh1, &L.dh2, &L.dra, &L.drb, &L.duh1, &L.da};
    for (float** p : nodes) al((void**)p, NH * 4);
    al((void**)&L.dgval, NG * 4);
    al((void**)&L.dgdiag, N * 4);
    float** vec[] = {&L.z, &L.v1, &L.v2};
    for (float** p : vec) al((void**)p, N * 4);
    al((void**)&L.loss, 4 * sizeof(double));
    cudaDeviceSynchronize();
    return ok ? MPS_OK : MPS_ERR_CUDA;
}

void lp_free(LearnedWork& L) {
    void* ps[] = {L.s_cnt, L.s_col, L.s_val, L.s_diag,
                  L.w32, L.w16, L.grad, L.adam_m, L.adam_v, L.scols, L.scnt, L.nlow, L.gdiag, L.gval,
                  L.a1,  L.pre1, L.h1,  L.uh1,  L.a2,  L.pre2, L.h2,  L.ra,   L.rb,  L.dgpre, L.dinv,
                  L.dh1, L.dh2, L.dra,  L.drb,  L.duh1, L.da,  L.dgval, L.dgdiag, L.z, L.v1, L.v2,
                  L.loss};
    for (void* p : ps)
        if (p) cudaFree(p);
    L = LearnedWork();
}

// Initial parameters: small random weights (splitmix64 uniform, scaled by
// 1/sqrt(fan-in)), readout weights om = 0 and bd = log(e - 1 - GMIN), so the
// initial factor is G = I: the preconditioner starts as diagonal scaling.
void lp_init_params(float* w, uint64_t seed) {
    uint64_t s = seed * 0x9E3779B97F4A7C15ull + 1;
    auto uni = [&]() {
        s += 0x9E3779B97F4A7C15ull;
        uint64_t z = s;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
    };
    memset(w, 0, sizeof(float) * LP_NPARAM);
    auto fill = [&](int off, int n, double scale) {
        for (int k = 0; k < n; k++) w[off + k] = (float)(scale * uni());
    };
    fill(LP_W1E, LP_H * LP_F, 1.0 / std::sqrt((double)LP_F));
    fill(LP_V1, LP_H * LP_H, 1.0 / 8.0);
    fill(LP_W2E, LP_H * LP_F, 1.0 / std::sqrt((double)LP_F));
    fill(LP_U2, LP_H * LP_H, 1.0 / 8.0);
    fill(LP_V2, LP_H * LP_H, 1.0 / 8.0);
    fill(LP_RE, LP_H * LP_F, 1.0 / std::sqrt((double)LP_F));
    fill(LP_RA, LP_H * LP_H, 1.0 / 8.0);
    fill(LP_RB, LP_H * LP_H, 1.0 / 8.0);
    fill(LP_DL, LP_H, 0.0);
    w[LP_BD] = (float)std::log(std::exp(1.0 - LP_GMIN) - 1.0);
}

void lp_upload_params(LearnedWork& L, const float* w, cudaStream_t st) {
    cudaMemcpyAsync(L.w32, w, LP_NPARAM * 4, cudaMemcpyHostToDevice, st);
    k_lp_to_bf16<<<blocks_for(LP_NPARAM, 256), 256, 0, st>>>(L.w32, L.w16, LP_NPARAM);
    cudaMemsetAsync(L.adam_m, 0, LP_NPARAM * 4, st);
    cudaMemsetAsync(L.adam_v, 0, LP_NPARAM * 4, st);
    L.adam_t = 0;
}

static FwdArgs fwd_args(LearnedWork& L, const LpSystem& S) {
    FwdArgs A;
    A.S = S;
    A.scols = L.scols;
    A.scnt = L.scnt;
    A.nlow = L.nlow;
    A.w = L.w16;
    A.a1 = L.a1;
    A.a2 = L.a2;
    A.uh1 = L.uh1;
    A.ra = L.ra;
    A.rb = L.rb;
    A.h2 = L.h2;
    A.gval = L.gval;
    A.gdiag = L.gdiag;
    A.dgpre = L.dgpre;
    return A;
}

void lp_build_stencil(LearnedWork& L, const LpSystem& S, uint32_t cap, cudaStream_t st) {
    k_lp_stencil<<<blocks_for(cap * 32u, 256), 256, 0, st>>>(S, L.scols, L.scnt, L.nlow, L.dinv,
                                                             const_cast<Scalars*>(S.sc));
}

// Grids of the tensor-core kernels: one resident wave of k_lp_dense_tc (it
// loops over the tiles) and two CTAs an SM for k_lp_wgrad_tc (few partial
// accumulators to add up, enough loads in flight).
struct TcGrids {
    uint32_t dense, wgrad;
};
static TcGrids tc_grids(uint32_t cap) {
    static uint32_t resident = 0, sms_seen = 0;
    if (resident == 0) {
        cudaFuncSetAttribute(k_lp_dense_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM);
        cudaFuncSetAttribute(k_lp_wgrad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TW_SMEM);
        int per_sm = 0, dev = 0, sms = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_lp_dense_tc, TC_M, TC_SMEM);
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        sms_seen = (uint32_t)(sms > 0 ? sms : 148);
        resident = (uint32_t)(per_sm > 0 ? per_sm : 1) * sms_seen;
    }
    const uint32_t t = blocks_for(cap, TC_M), w = blocks_for(cap, TW_K);
    return TcGrids{t < resident ? t : resident, w < 2 * sms_seen ? w : 2 * sms_seen};
}

void lp_forward(LearnedWork& L, const LpSystem& S, bool exact, uint32_t cap, cudaStream_t st, bool tensor_cores,
                bool keep_pre) {
    (void)exact;
    const uint32_t wb = blocks_for(cap * 32u, 256);   // warp per row
    const uint32_t db = blocks_for(cap, 4);           // 4 rows per dense block
    const uint32_t dgrid = db < 148u * 8u ? db : 148u * 8u;
    const uint32_t tgrid = tensor_cores ? tc_grids(cap).dense : 0u;
    uint32_t* err = const_cast<uint32_t*>(&S.sc->err);
    auto dense = [&](const float* x, int woff, int boff, const float* resid, float* pre, float* out, int act) {
        if (tensor_cores)  // the pre-activations feed nothing but the backward pass
            k_lp_dense_tc<<<tgrid, TC_M, TC_SMEM, st>>>(x, L.w16, woff, boff, resid, keep_pre ? pre : nullptr, out,
                                                        act, S.rowlist, S.nrows, err, 0, 0);
        else
            k_lp_dense_fwd<<<dgrid, 256, 0, st>>>(x, L.w16, woff, boff, resid, pre, out, act, S.rowlist, S.nrows);
    };
    FwdArgs A = fwd_args(L, S);
    k_lp_edge_fwd<1><<<wb, 256, 0, st>>>(A);
    dense(L.a1, LP_V1, LP_C1, nullptr, L.pre1, L.h1, 1);
    dense(L.h1, LP_U2, -1, nullptr, nullptr, L.uh1, 0);
    k_lp_edge_fwd<2><<<wb, 256, 0, st>>>(A);
    dense(L.a2, LP_V2, LP_C2, L.h1, L.pre2, L.h2, 1);
    dense(L.h2, LP_RA, -1, nullptr, nullptr, L.ra, 0);
    dense(L.h2, LP_RB, -1, nullptr, nullptr, L.rb, 0);
    k_lp_readout_fwd<<<wb, 256, 0, st>>>(A);
    k_lp_transpose<<<blocks_for(cap, 256), 256, 0, st>>>(L.scols, L.scnt, L.nlow, L.gval, S.rowlist, S.nrows);
}

// ---------------------------------------------------------------- symmetric form
__global__ void k_lp_sym_reset(uint32_t* __restrict__ s_cnt, float* __restrict__ s_diag, uint32_t n) {
    const uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    s_cnt[id] = 0;
    s_diag[id] = 1.f;
}

// Row i (thread per row): S_ij = G_ii G_ij for its j < i entries and
// G_ji G_jj for its j > i ones (k_lp_transpose left G_ji there); the two
// products of one pair are the same two factors, so S is symmetric bit for
// bit.  S_ii = max(G_ii^2, (1 + 1e-2) sum_j |S_ij|).
__global__ void __launch_bounds__(256) k_lp_sym_build(LpSystem S, const uint32_t* __restrict__ scols,
                                                      const uint32_t* __restrict__ scnt,
                                                      const uint32_t* __restrict__ nlow, const float* __restrict__ gval,
                                                      const float* __restrict__ gdiag, uint32_t* __restrict__ s_cnt,
                                                      uint32_t* __restrict__ s_col, float* __restrict__ s_val,
                                                      float* __restrict__ s_diag) {
    const uint32_t R = *S.nrows;
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= R) return;
    const uint32_t i = __ldg(S.rowlist + k);
    const uint32_t id = __ldg(S.id + i);
    const float gi = gdiag[i];
    const uint32_t n = scnt[i], nl = nlow[i];
    float sum = 0.f;
    for (uint32_t t = 0; t < n; t++) {
        const uint32_t j = scols[(size_t)i * LP_GW + t];
        const float g = gval[(size_t)i * LP_GW + t];
        const float v = t < nl ? gi * g : g * gdiag[j];
        s_col[(size_t)id * LP_GW + t] = __ldg(S.id + j);
        s_val[(size_t)id * LP_GW + t] = v;
        sum += fabsf(v);
    }
    s_cnt[id] = n;
    s_diag[id] = fmaxf(gi * gi, 1.01f * sum);  // the margin covers the solver's BF16 off-diagonals
}

int lp_alloc_symmetric(LearnedWork& L) {
    if (L.s_cnt) return MPS_OK;
    const size_t N = L.cap, NG = (size_t)L.cap * LP_GW;
    if (cudaMalloc(&L.s_cnt, N * 4 + 64) != cudaSuccess || cudaMalloc(&L.s_col, NG * 4 + 64) != cudaSuccess ||
        cudaMalloc(&L.s_val, NG * 4 + 64) != cudaSuccess || cudaMalloc(&L.s_diag, N * 4 + 64) != cudaSuccess)
        return MPS_ERR_CUDA;
    return MPS_OK;
}

int lp_build_symmetric(LearnedWork& L, const LpSystem& S, uint32_t np0, cudaStream_t st) {
    if (!L.s_cnt) return MPS_ERR_INVALID;
    k_lp_sym_reset<<<blocks_for(np0, 256), 256, 0, st>>>(L.s_cnt, L.s_diag, np0);
    k_lp_sym_build<<<blocks_for(L.cap, 256), 256, 0, st>>>(S, L.scols, L.scnt, L.nlow, L.gval, L.gdiag, L.s_cnt,
                                                           L.s_col, L.s_val, L.s_diag);
    L.s_ready = true;
    return MPS_OK;
}

int lp_loss_grad(LearnedWork& L, const LpSystem& S, bool exact, uint64_t seed, uint32_t cap, cudaStream_t st) {
    if (lp_setup_training(L) != MPS_OK) return MPS_ERR_CUDA;
    // the stencil of this system (a step may have kept an older one between
    // network evaluations)
    lp_build_stencil(L, S, cap, st);
    // training: FP32 activations on the CUDA cores (the oracle's network), or
    // the 64 -> 64 layers' forward, dx and dW products on the tensor cores
    const bool tc = L.train_tensor_cores;
    lp_forward(L, S, exact, cap, st, tc, true);
    const uint32_t tb = blocks_for(cap, 256), wb = blocks_for(cap * 32u, 256);
    const uint32_t db = blocks_for(cap, 4);
    const uint32_t dgrid = db < 148u * 8u ? db : 148u * 8u;
    const TcGrids tg = tc ? tc_grids(cap) : TcGrids{0u, 0u};
    uint32_t* err = const_cast<uint32_t*>(&S.sc->err);
    // dx (+)= W^T dy, grad(W) += dy x^T, grad(b) += dy (boff >= 0)
    auto dense_bwd = [&](const float* dy, const float* x, int woff, float* dx, int accumulate, int boff) {
        if (tc) {
            k_lp_dense_tc<<<tg.dense, TC_M, TC_SMEM, st>>>(dy, L.w16, woff, -1, nullptr, nullptr, dx, 0, S.rowlist,
                                                           S.nrows, err, 1, accumulate);
            k_lp_wgrad_tc<<<tg.wgrad, TW_THREADS, TW_SMEM, st>>>(dy, x, woff, boff, L.grad, S.rowlist, S.nrows,
                                                                 err);
        } else {
            k_lp_dense_bwd<<<dgrid, 256, 0, st>>>(dy, x, L.w16, woff, dx, accumulate, L.grad, boff, S.rowlist,
                                                  S.nrows);
        }
    };
    cudaMemsetAsync(L.grad, 0, LP_NPARAM * 4, st);
    cudaMemsetAsync(L.loss, 0, 4 * sizeof(double), st);
    // Kaporin's condition number of G Ahat G^T with a Rademacher probe z:
    // v1 = G^T z, v2 = Ahat v1, T = v1 . v2
    k_lp_probe<<<tb, 256, 0, st>>>(S.id, L.z, seed, S.rowlist, S.nrows);
    k_lp_gapply<<<tb, 256, 0, st>>>(L.scols, L.scnt, L.nlow, L.gval, L.gdiag, L.z, L.v1, 1, S.rowlist, S.nrows);
    if (exact) k_lp_ahat<true><<<wb, 256, 0, st>>>(S, L.dinv, L.v1, L.v2);
    else k_lp_ahat<false><<<wb, 256, 0, st>>>(S, L.dinv, L.v1, L.v2);
    k_lp_kaporin<<<tb, 256, 0, st>>>(L.v1, L.v2, L.gdiag, L.loss, S.rowlist, S.nrows);
    k_lp_dg<<<tb, 256, 0, st>>>(L.scols, L.nlow, L.v2, L.z, L.gdiag, L.loss, L.dgval, L.dgdiag, S.rowlist, S.nrows);
    k_lp_transpose<<<tb, 256, 0, st>>>(L.scols, L.scnt, L.nlow, L.dgval, S.rowlist, S.nrows);
    // network backward
    BwdArgs B;
    B.S = S;
    B.scols = L.scols;
    B.scnt = L.scnt;
    B.nlow = L.nlow;
    B.w = L.w16;
    B.a1 = L.a1;
    B.pre1 = L.pre1;
    B.h1 = L.h1;
    B.uh1 = L.uh1;
    B.a2 = L.a2;
    B.pre2 = L.pre2;
    B.h2 = L.h2;
    B.ra = L.ra;
    B.rb = L.rb;
    B.dgpre = L.dgpre;
    B.dgval = L.dgval;
    B.dgdiag = L.dgdiag;
    B.dra = L.dra;
    B.drb = L.drb;
    B.dh2 = L.dh2;
    B.da = L.da;
    B.grad = L.grad;
    k_lp_readout_bwd_a<<<wb, 256, 0, st>>>(B);
    k_lp_readout_bwd_b<<<wb, 256, 0, st>>>(B);
    dense_bwd(L.dra, L.h2, LP_RA, L.dh2, 1, -1);
    dense_bwd(L.drb, L.h2, LP_RB, L.dh2, 1, -1);
    // second message pass, node: h2 = GELU(pre2) + h1
    const uint32_t eb = blocks_for(cap * (uint32_t)LP_H, 256);
    k_lp_copy_rows<<<eb, 256, 0, st>>>(L.dh2, L.dh1, S.rowlist, S.nrows);
    k_lp_gelu_bwd<<<eb, 256, 0, st>>>(L.dh2, L.pre2, L.dra, S.rowlist, S.nrows);  // dra reused as dpre2
    dense_bwd(L.dra, L.a2, LP_V2, L.da, 0, LP_C2);
    k_lp_edge_bwd_a<2><<<wb, 256, 0, st>>>(B);
    k_lp_edge2_bwd_b<<<wb, 256, 0, st>>>(B, L.duh1);
    dense_bwd(L.duh1, L.h1, LP_U2, L.dh1, 1, -1);
    // first message pass, node: h1 = GELU(pre1)
    k_lp_gelu_bwd<<<eb, 256, 0, st>>>(L.dh1, L.pre1, L.dra, S.rowlist, S.nrows);  // dpre1
    dense_bwd(L.dra, L.a1, LP_V1, L.da, 0, LP_C1);
    k_lp_edge_bwd_a<1><<<wb, 256, 0, st>>>(B);
    return MPS_OK;
}

double lp_loss_value(const double* sums, uint32_t nrows) {
    if (nrows == 0 || !(sums[0] > 0.0)) return 0.0;
    const double n = (double)nrows;
    return std::log(sums[0] / n) - 2.0 * sums[1] / n;
}

void lp_adam(LearnedWork& L, float lr, cudaStream_t st) {
    L.adam_t++;
    const float b1c = 1.f - std::pow(0.9f, (float)L.adam_t), b2c = 1.f - std::pow(0.999f, (float)L.adam_t);
    k_lp_adam<<<blocks_for(LP_NPARAM, 256), 256, 0, st>>>(L.w32, L.w16, L.grad, L.adam_m, L.adam_v, LP_NPARAM, lr,
                                                          b1c, b2c);
}

}  // namespace mpsb
