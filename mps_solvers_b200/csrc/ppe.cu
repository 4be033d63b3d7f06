// ppe.cu -- assembly and persistent CG solve of the pressure Poisson equation.
//
// The reference builds a dense np x np matrix and runs CG with cuBLAS gemv/dot
// calls driven from the host, one host sync per dot product
// (MPS_CAL_v4.0/cuda_ker.cu:171-297), or a dense CPU CG
// (MPS_CAL_v4.0/MPS_CPU.cpp:829-888).  Here the matrix holds only the
// neighbour stencil, and the whole solve is one cooperative kernel:
//
//   outer (defect correction, FP64): r64 = b - A x64; stop when
//       |r64| <= tol |b| (FP64 norms of the true residual)
//   inner (FP32 vectors, FP64 dot products): Jacobi-preconditioned CG on
//       A d = r64 from d = 0 until |r| <= eta |r64|, with x64 += alpha p
//       accumulated in FP64 as it goes.
//
// Grid-wide reductions are fused with a counter + generation barrier with a
// bounded spin: a barrier that does not complete within ~1 s sets
// ERR_DEVICE_TIMEOUT and the kernel returns.  Partial sums are added in a
// fixed order, so the solve is bit-reproducible for a given device and grid.
#include <cstring>
#include <vector>

#include "cellsort.cuh"
#include "ppe.cuh"
#include "ppe_device.cuh"

namespace mpsb {

static inline uint32_t blocks_for(uint32_t n, uint32_t t) { return (n + t - 1) / t; }

// ---------------------------------------------------------------- assembly
struct AsmArgs {
    StageArgs a;
    uint32_t* cols;
    float* wrm;              // the entries' weights, beside cols
    uint32_t* rlen;
    double* diag64;
    float* diag32;
    float* inv_diag;
    double* b64;
    double* x64;
    unsigned* bar;
    double n0, lambda, beta, b_tmp, rho_lambda_alpha_n0, dim2;
    const PpeScene* scenes;  // per scene of a batch (these constants otherwise)
};

// One warp per particle: scan the reference's 27 linked cells for rlap
// neighbours of type != 2, accumulate the diagonal, append the non-Dirichlet
// ones in ascending index order (MPS_CAL_v4.0/MPS_CPU.cpp:651-698).
template <bool EX, bool BT>
__global__ void __launch_bounds__(256) k_ppe_assemble(AsmArgs A) {
    const StageArgs& a = A.a;
    const uint32_t n = a.sc->np;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (blockIdx.x == 0 && threadIdx.x == 0) A.bar[0] = 0u;  // the solver's barrier starts empty
    if (i >= n) return;
    const float4* __restrict__ pos = a.cur.pos;
    const float* __restrict__ nn = a.cur.n;
    const float4 pi = pos[i];
    const double ni = (double)nn[i];
    const Local L = local_of<BT>(a, i);
    double n0 = A.n0, beta = A.beta, b_tmp = A.b_tmp, rlan0 = A.rho_lambda_alpha_n0;
    if (BT) {
        const PpeScene& ps = A.scenes[L.s];
        n0 = ps.n0;
        beta = ps.beta;
        b_tmp = ps.b_tmp;
        rlan0 = ps.rho_lambda_alpha_n0;
    }
    const bool dir_i = ptype(pi) == T_DUMMY || ni < beta * n0;
    if (dir_i) {
        if (lane == 0) {
            A.rlen[i] = PPE_DIRICHLET;
            A.diag64[i] = 1.0;
            A.diag32[i] = 1.0f;
            A.inv_diag[i] = 1.0f;
            A.b64[i] = 0.0;
            A.x64[i] = 0.0;
        }
        return;
    }
    const double dt = (double)dt_of<BT>(a, L.s);
    const double Aii = rlan0 / (A.dim2 * dt * dt);
    const Phys P = phys_of<BT>(a, L.s);
    const float re = P.rlap, thr = P.rlap_thr;
    const double bthr = beta * n0;
    // n_j < bthr (double) exactly when n_j < bthr_f, the least float >= bthr
    float bthr_f = (float)bthr;
    if ((double)bthr_f < bthr) bthr_f = nextafterf(bthr_f, INFINITY);
    uint32_t* cols = A.cols + (size_t)i * PPE_W;
    float* wrow = A.wrm + (size_t)i * PPE_W;
    uint32_t count = 0;
    float diag_lane = 0.f;  // this lane's few nonzero weights, then a FP64 warp sum
    const uint32_t lt = (1u << lane) - 1u;
    const CellNear nr = cell_near(L.g, L.c, pi.x, pi.y, pi.z, re);
    walk_cells<!EX>(L.g, L.cs, L.c, nr, lane, [&](uint32_t j, bool in) {
        {
            bool app = false;
            float w = 0.f;
            if (in && j != i) {
                const float4 pj = __ldg(pos + j);
                if (ptype(pj) != T_DUMMY) {
                    const float dx = fsub<EX>(pj.x, pi.x), dy = fsub<EX>(pj.y, pi.y), dz = fsub<EX>(pj.z, pi.z);
                    const float rr = dot3<EX>(dx, dy, dz, dx, dy, dz);
                    if (rr < thr) {
                        w = weight_rr<EX>(re, rr);
                        if (w > 0.f) app = !(__ldg(nn + j) < bthr_f);
                    }
                }
            }
            diag_lane += w;
            const uint32_t m = __ballot_sync(0xffffffffu, app);
            if (app) {
                const uint32_t k = count + __popc(m & lt);
                if (k < PPE_W) {
                    cols[k] = j;
                    wrow[k] = w;
                }
            }
            count += __popc(m);
        }
    });
    const double diag = warp_sum_d((double)diag_lane);
    if (lane == 0) {
        if (count > PPE_W) {
            atomicOr(&a.sc->err, ERR_CAPACITY);  // more than PPE_W neighbours
            count = PPE_W;
        }
        const double dg = -diag - Aii;
        A.rlen[i] = count;
        A.diag64[i] = dg;
        A.diag32[i] = (float)dg;
        A.inv_diag[i] = (float)(1.0 / dg);
        A.b64[i] = b_tmp * (n0 - ni);
        A.x64[i] = (double)a.cur.press[i];
    }
}

// ---------------------------------------------------------------- solve
struct SolveArgs {
    const uint32_t* cols;
    const uint32_t* rlen;
    const double* diag64;
    const float* diag32;
    const float* inv_diag;
    const double* b64;
    double* x64;
    float* r;
    float2* zp0;   // (z, p) per row, two buffers: current and next
    float2* zp1;
    float* q;
    float* qp;        // the product's row sums of slice parts 1 .. PPE_MAX_SPLIT - 1
    uint32_t cap;
    double* part;
    double* result;
    unsigned* bar;
    const uint32_t* rowlist;
    const uint32_t* nrows;
    const uint32_t* off;
    const uint32_t* scols;
    const float* sw;          // stored weights (same layout as scols)
    const float4* pos;
    float rlap, rlap_thr;
    // learned preconditioner S' by particle columns (ppe_device.cuh), and
    // its residual and q interleaved per particle, current and next pair
    // buffer (a neighbour's r - alpha q is one 8-byte load)
    const uint32_t* sp_off;
    const uint32_t* sp_ent;
    const float* sp_diag;
    float2* rq0;
    float2* rq1;
    Scalars* sc;
    double tol;
    double eta_min;   // smallest inner reduction asked of one FP32 solve
    uint32_t keep;    // matrix entries read as evict_last (mat_policy)
    int max_iter;
    int inner_cap;
    int max_outer;
    int smem_chunks;  // stored weights: each warp's last chunks held in shared memory
};

// The weight of a stored neighbour, recomputed from the positions with the
// function the assembly used for the diagonal (so the operator is the same
// matrix in every product); a padding entry (j == i) weighs 0.
template <bool EX>
__device__ __forceinline__ float stencil_weight(const SolveArgs& S, const float4& pi, uint32_t i, uint32_t j) {
    const float4 pj = __ldg(S.pos + j);
    const float dx = fsub<EX>(pj.x, pi.x), dy = fsub<EX>(pj.y, pi.y), dz = fsub<EX>(pj.z, pi.z);
    const float rr = dot3<EX>(dx, dy, dz, dx, dy, dz);
    return (j != i && rr < S.rlap_thr) ? weight_rr<EX>(S.rlap, rr) : 0.f;
}

// The weights of one lane's 4 entries: stored, or recomputed from positions.
template <bool EX, bool SW>
__device__ __forceinline__ float4 chunk_weights(const float4* __restrict__ w4, uint64_t pol,
                                                const float4* __restrict__ pos, float rlap, float thr,
                                                const float4& pi, uint32_t i, const uint4& c) {
    if (SW) return ld_mat(w4, pol);
    auto one = [&](uint32_t j) {
        const float4 pj = __ldg(pos + j);
        const float dx = fsub<EX>(pj.x, pi.x), dy = fsub<EX>(pj.y, pi.y), dz = fsub<EX>(pj.z, pi.z);
        const float rr = dot3<EX>(dx, dy, dz, dx, dy, dz);
        return (j != i && rr < thr) ? weight_rr<EX>(rlap, rr) : 0.f;
    };
    return make_float4(one(c.x), one(c.y), one(c.z), one(c.w));
}

// SW: stored weights (the pack's) instead of recomputing them from the
// positions; the two give the same matrix, the autotuner picks the faster.
// Parts per slice of the CG product: 1 while there are at least as many
// slices as warps (measured best at 310,912 particles), else enough parts to
// give every warp work, at most PPE_MAX_SPLIT (33,072 particles: 0.63 ms ->
// 0.47 ms per solve with 4).
constexpr uint32_t PPE_MAX_SPLIT = 4;
__device__ __forceinline__ uint32_t ppe_split(uint32_t nslices, uint32_t nwarps) {
    if (nslices == 0 || nslices >= nwarps) return 1u;
    const uint32_t p = (nwarps + nslices - 1) / nslices;
    return p < PPE_MAX_SPLIT ? p : PPE_MAX_SPLIT;
}

// q_i of the last product: part 0's value plus the other parts' row sums,
// added in part order
__device__ __forceinline__ float q_total(const SolveArgs& S, uint32_t i, uint32_t parts) {
    float v = S.q[i];
    for (uint32_t p = 1; p < parts; p++) v += S.qp[(size_t)(p - 1) * S.cap + i];
    return v;
}

// the learned form: r_j - alpha q_j from the (r, q) pairs, q_j added up over
// the parts in the same order as q_total
__device__ __forceinline__ float rq_next(const SolveArgs& S, const float2* rq, uint32_t j, uint32_t parts, float a) {
    const float2 v = rq[j];
    float qv = v.y;
    for (uint32_t p = 1; p < parts; p++) qv += S.qp[(size_t)(p - 1) * S.cap + j];
    return fmaf(-a, qv, v.x);
}

// PREC 0: diagonal scaling; PREC 1: the learned S' (particle columns), its
// product fused into the residual update with each neighbour's r - alpha q
// formed from the (r, q) pairs, the new residual into the other pair buffer;
// both keep two grid-wide reductions per iteration.
template <bool EX, int PREC, bool SW>
__global__ void __launch_bounds__(PPE_THREADS) k_ppe_solve(SolveArgs S) {
    // Rows are the ordered list of non-Dirichlet rows; slices of 8 of them
    // are dealt to warps round-robin (4 lanes per row inside a slice); the
    // row-wise vector updates take one thread per row.
    const uint32_t R = *S.nrows;
    const uint32_t nslices = (R + SELL_C - 1) / SELL_C;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t rsub = lane & 7, q = lane >> 3;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    const uint32_t parts = ppe_split(nslices, nw);
    const uint32_t* __restrict__ rowlist = S.rowlist;
    // With stored weights each warp keeps the last C chunks of its share of
    // the products (the same chunks in every product: the deal of work items
    // to warps is fixed) in shared memory for the whole solve; chunk g of
    // the warp's sequence comes from shared memory when g >= g0.
    extern __shared__ __align__(16) unsigned char sol_sm[];
    const uint32_t C = SW ? (uint32_t)S.smem_chunks : 0u;
    const uint32_t wib = threadIdx.x >> 5;
    uint4* smc = reinterpret_cast<uint4*>(sol_sm) + (size_t)wib * C * 32;
    float4* smw = reinterpret_cast<float4*>(sol_sm + (size_t)(blockDim.x >> 5) * C * 32 * sizeof(uint4)) +
                  (size_t)wib * C * 32;
    uint32_t g0 = 0xffffffffu;
    if (C) {
        uint32_t U = 0;
        for (uint32_t u = gw; u < parts * nslices; u += nw) {
            const uint32_t sl = u / parts, part = u % parts;
            const uint32_t T = (__ldg(S.off + sl + 1) - __ldg(S.off + sl)) >> 7;
            U += (part + 1) * T / parts - part * T / parts;
        }
        g0 = U > C ? U - C : 0u;
        uint32_t g = 0;
        for (uint32_t u = gw; u < parts * nslices; u += nw) {
            const uint32_t sl = u / parts, part = u % parts;
            const uint32_t base = __ldg(S.off + sl);
            const uint32_t T = (__ldg(S.off + sl + 1) - base) >> 7;
            const uint32_t t0 = part * T / parts, t1 = (part + 1) * T / parts;
            const uint4* cols = reinterpret_cast<const uint4*>(S.scols + base) + lane;
            const float4* wts = reinterpret_cast<const float4*>(S.sw + base) + lane;
            for (uint32_t t = t0; t < t1; t++, g++)
                if (g >= g0) {
                    smc[(g - g0) * 32 + lane] = __ldg(cols + 32 * t);
                    smw[(g - g0) * 32 + lane] = __ldg(wts + 32 * t);
                }
        }
        __syncwarp();
    }
    int total = 0, outers = 0;
    double relres = 0.0;
    bool converged = false;
    // (z, p) of every row, interleaved so that a neighbour's pair is one
    // 8-byte load; zc is read by the products, zn receives the next pair
    float2* zc = S.zp0;
    float2* zn = S.zp1;
    for (int outer = 0; outer < S.max_outer; outer++) {
        // ---- true residual r64 = b - A x64 (FP64), inner start: z = M^-1 r, p = 0
        double acc[3] = {0.0, 0.0, 0.0};  // |r64|^2, |b|^2, r.z
        for (uint32_t sl = gw; sl < nslices; sl += nw) {
            const uint32_t k = sl * SELL_C + rsub;
            const uint32_t base = __ldg(S.off + sl);
            const uint64_t pol = mat_policy(base, S.keep);
            const uint32_t T = (__ldg(S.off + sl + 1) - base) >> 7;  // chunks of 16 per row
            const uint4* cols = reinterpret_cast<const uint4*>(S.scols + base) + lane;
            const float4* wts = reinterpret_cast<const float4*>(S.sw + base) + lane;
            const uint32_t ii = k < R ? __ldg(rowlist + k) : 0u;
            const float4 pi = __ldg(S.pos + ii);
            double s = 0.0;
            for (uint32_t t = 0; t < T; t++) {
                const uint4 c = ld_mat(cols + 32 * t, pol);
                const float4 w = chunk_weights<EX, SW>(wts + 32 * t, pol, S.pos, S.rlap, S.rlap_thr, pi, ii, c);
                s += (double)w.x * S.x64[c.x] + (double)w.y * S.x64[c.y] + (double)w.z * S.x64[c.z] +
                     (double)w.w * S.x64[c.w];
            }
            s += __shfl_xor_sync(0xffffffffu, s, 8);
            s += __shfl_xor_sync(0xffffffffu, s, 16);
            if (q == 0 && k < R) {
                const uint32_t i = __ldg(rowlist + k);
                const double bi = S.b64[i];
                const double ri = bi - (S.diag64[i] * S.x64[i] + s);
                const float rf = (float)ri;
                if (PREC == 1) S.rq0[i].x = rf;
                else S.r[i] = rf;
                acc[0] += ri * ri;
                acc[1] += bi * bi;
                if (PREC == 0) {
                    const float zf = rf * S.inv_diag[i];
                    zc[i] = make_float2(zf, 0.f);
                    acc[2] += (double)rf * (double)zf;
                } else {
                    zc[i].y = 0.f;
                }
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
        if (PREC == 1) {
            // z = S' r of the new residual, r.z
            double rzp[1] = {0.0};
            const float2* rq = S.rq0;
            for (uint32_t kk = blockIdx.x * blockDim.x + threadIdx.x; kk < R; kk += gridDim.x * blockDim.x) {
                const uint32_t i = __ldg(rowlist + kk);
                const float zi =
                    sp_row_at(S.sp_off, S.sp_ent, S.sp_diag, kk, i, [rq](uint32_t j) { return rq[j].x; });
                zc[i].x = zi;
                rzp[0] += (double)rq[i].x * (double)zi;
            }
            double tz[1];
            if (!grid_reduce<1>(rzp, S.part, S.result, S.bar, S.sc, tz)) return;
            tot[2] = tz[0];
        }
        // inner target |r| <= eta |r64|
        double eta = 0.3 * S.tol / relres;
        if (eta < S.eta_min) eta = S.eta_min;
        if (eta > 0.5) eta = 0.5;
        const double stop = eta * eta * rr64;
        double rz = tot[2];
        float beta = 0.f;
        for (int it = 0; it < S.inner_cap && total < S.max_iter; it++) {
            // ---- q = A p_new with p_new = z + beta p (fused), p.q.  Work
            // items are parts of a slice (`parts` chunk ranges), so that all
            // warps have work when there are fewer slices than warps; part 0
            // adds the diagonal and writes q, part p > 0 writes its row sums
            // to qp[p - 1], and p.q adds every part's p_i * (its share of
            // q_i), which is linear in the shares.
            double pq[1] = {0.0};
            uint32_t g = 0;  // this warp's chunks so far (the shared-memory tail)
            for (uint32_t u = gw; u < parts * nslices; u += nw) {
                const uint32_t sl = u / parts, part = u % parts;
                const uint32_t k = sl * SELL_C + rsub;
                const uint32_t base = __ldg(S.off + sl);
                const uint64_t pol = mat_policy(base, S.keep);
                const uint32_t T = (__ldg(S.off + sl + 1) - base) >> 7;  // chunks of 16 per row
                const uint32_t t0 = part * T / parts, t1 = (part + 1) * T / parts;
                // chunks [ts, t1) of this item come from shared memory
                const uint32_t ts = g >= g0 ? t0 : (g0 - g >= t1 - t0 ? t1 : t0 + (g0 - g));
                const uint4* cols = reinterpret_cast<const uint4*>(S.scols + base) + lane;
                const float4* wts = reinterpret_cast<const float4*>(S.sw + base) + lane;
                const uint32_t ii = k < R ? __ldg(rowlist + k) : 0u;
                const float4 pi = __ldg(S.pos + ii);
                float s0 = 0.f, s1 = 0.f;
#pragma unroll 4  // measured: 4 chunks per step beat 2 (and a cp.async ring)
                for (uint32_t t = t0; t < ts; t++) {
                    const uint4 c = ld_mat(cols + 32 * t, pol);
                    const float4 w = chunk_weights<EX, SW>(wts + 32 * t, pol, S.pos, S.rlap, S.rlap_thr, pi, ii, c);
                    const float2 a0 = zc[c.x], a1 = zc[c.y], a2 = zc[c.z], a3 = zc[c.w];
                    s0 = fmaf(w.x, fmaf(beta, a0.y, a0.x), s0);
                    s1 = fmaf(w.y, fmaf(beta, a1.y, a1.x), s1);
                    s0 = fmaf(w.z, fmaf(beta, a2.y, a2.x), s0);
                    s1 = fmaf(w.w, fmaf(beta, a3.y, a3.x), s1);
                }
                if (SW) {
                    const uint32_t gs = g + (ts - t0) - g0;  // shared-memory slot of chunk ts
#pragma unroll 2
                    for (uint32_t t = ts; t < t1; t++) {
                        const uint4 c = smc[(gs + t - ts) * 32 + lane];
                        const float4 w = smw[(gs + t - ts) * 32 + lane];
                        const float2 a0 = zc[c.x], a1 = zc[c.y], a2 = zc[c.z], a3 = zc[c.w];
                        s0 = fmaf(w.x, fmaf(beta, a0.y, a0.x), s0);
                        s1 = fmaf(w.y, fmaf(beta, a1.y, a1.x), s1);
                        s0 = fmaf(w.z, fmaf(beta, a2.y, a2.x), s0);
                        s1 = fmaf(w.w, fmaf(beta, a3.y, a3.x), s1);
                    }
                }
                g += t1 - t0;
                float s = s0 + s1;
                s += __shfl_xor_sync(0xffffffffu, s, 8);
                s += __shfl_xor_sync(0xffffffffu, s, 16);
                if (q == 0 && k < R) {
                    const uint32_t i = __ldg(rowlist + k);
                    const float2 o = zc[i];
                    const float pn = fmaf(beta, o.y, o.x);
                    float qi = s;
                    if (part == 0) {
                        qi = fmaf(S.diag32[i], pn, s);
                        zn[i].y = pn;
                        if (PREC == 1) S.rq0[i].y = qi;
                        else S.q[i] = qi;
                    } else {
                        S.qp[(size_t)(part - 1) * S.cap + i] = s;
                    }
                    pq[0] += (double)pn * (double)qi;
                }
            }
            double totp[1];
            if (!grid_reduce<1>(pq, S.part, S.result, S.bar, S.sc, totp)) return;
            const double alpha = rz / totp[0];
            const float alpha_f = (float)alpha;
            // ---- x64 += alpha p, r -= alpha q, z = M^-1 r, r.z, r.r
            double acc2[2] = {0.0, 0.0};
            double tot2[2];
            if (PREC == 0) {
                for (uint32_t kk = blockIdx.x * blockDim.x + threadIdx.x; kk < R; kk += gridDim.x * blockDim.x) {
                    const uint32_t i = __ldg(rowlist + kk);
                    const float pn = zn[i].y;
                    S.x64[i] += alpha * (double)pn;
                    const float ri = fmaf(-alpha_f, q_total(S, i, parts), S.r[i]);
                    const float zi = ri * S.inv_diag[i];
                    S.r[i] = ri;
                    zn[i] = make_float2(zi, pn);
                    acc2[0] += (double)ri * (double)zi;
                    acc2[1] += (double)ri * (double)ri;
                }
                if (!grid_reduce<2>(acc2, S.part, S.result, S.bar, S.sc, tot2)) return;
            } else {
                // z = S' r_new with each neighbour's r_new = r - alpha q formed
                // on the fly; the new residual into the second buffer (the
                // neighbours read the old one); r.z and r.r
                float2* rnew = S.rq1;
                const float2* rq = S.rq0;
                const SolveArgs& SS = S;
                for (uint32_t kk = blockIdx.x * blockDim.x + threadIdx.x; kk < R; kk += gridDim.x * blockDim.x) {
                    const uint32_t i = __ldg(rowlist + kk);
                    const float pn = zn[i].y;
                    S.x64[i] += alpha * (double)pn;
                    const float ri = rq_next(S, rq, i, parts, alpha_f);
                    rnew[i] = make_float2(ri, 0.f);
                    const float zi = sp_row_at(S.sp_off, S.sp_ent, S.sp_diag, kk, i,
                                               [rq, &SS, alpha_f, parts](uint32_t j) {
                                                   return rq_next(SS, rq, j, parts, alpha_f);
                                               });
                    zn[i] = make_float2(zi, pn);
                    acc2[0] += (double)ri * (double)zi;
                    acc2[1] += (double)ri * (double)ri;
                }
                if (!grid_reduce<2>(acc2, S.part, S.result, S.bar, S.sc, tot2)) return;
                // swap the pair buffers
                S.rq1 = S.rq0;
                S.rq0 = rnew;
            }
            total++;
            beta = (float)(tot2[0] / rz);
            rz = tot2[0];
            float2* t = zc;
            zc = zn;
            zn = t;
            if (tot2[1] <= stop) break;
        }
        // the last inner iteration ended on a grid-wide reduction, so every
        // x64 update is visible to the residual pass of the next round
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        S.sc->cg_iters = total;
        S.sc->cg_outer = outers;
        S.sc->cg_relres = relres;
        if (!converged) atomicOr(&S.sc->err, ERR_CG_NOT_CONVERGED);
    }
}

// ---------------------------------------------------------------- pipelined solve
// Diagonally scaled PCG in the pipelined form of Ghysels and Vanroose (2014)
// with the recurrences of Chronopoulos and Gear: per iteration one product
// n = A m (m = M w) and one grid-wide reduction of (r.u, w.u, r.r), where
// the standard form needs two reductions.  Algebraically the same iterates
// as PCG; in floating point the recursive residual drifts more, which the
// FP64 true-residual passes absorb (the solve still ends on
// |b - A x| <= tol |b| in FP64).  The neighbours' m_j = M w_j are read from a
// double buffer written by the previous iteration, one 4-byte load each.
struct PipeArgs {
    const uint32_t* rowlist;
    const uint32_t* nrows;
    const uint32_t* off;
    const uint32_t* scols;
    const float* sw;
    const float4* pos;
    float rlap, rlap_thr;
    const double* b64;
    const double* diag64;
    const float* diag32;
    const float* inv_diag;
    double* x64;
    float *r, *u, *w, *z, *q, *s, *p;
    float *m0, *m1;
    double* part;
    double* result;
    unsigned* bar;
    Scalars* sc;
    double tol, eta_min;
    uint32_t keep;
    int max_iter, inner_cap, max_outer;
};

template <bool EX, bool SW>
__global__ void __launch_bounds__(PPE_THREADS) k_ppe_solve_pipe(PipeArgs S) {
    const uint32_t R = *S.nrows;
    const uint32_t nslices = (R + SELL_C - 1) / SELL_C;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t rsub = lane & 7, q = lane >> 3;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    const uint32_t* __restrict__ rowlist = S.rowlist;
    int total = 0, outers = 0;
    double relres = 0.0;
    bool converged = false;
    float* mc = S.m0;   // m = M w read by this iteration's product
    float* mn = S.m1;   // m of the next iteration
    for (int outer = 0; outer < S.max_outer; outer++) {
        // ---- FP64 true residual; r, u = M r
        double acc[2] = {0.0, 0.0};  // |r64|^2, |b|^2
        for (uint32_t sl = gw; sl < nslices; sl += nw) {
            const uint32_t k = sl * SELL_C + rsub;
            const uint32_t base = __ldg(S.off + sl);
            const uint64_t pol = mat_policy(base, S.keep);
            const uint32_t T = (__ldg(S.off + sl + 1) - base) >> 7;
            const uint4* cols = reinterpret_cast<const uint4*>(S.scols + base) + lane;
            const float4* wts = reinterpret_cast<const float4*>(S.sw + base) + lane;
            const uint32_t ii = k < R ? __ldg(rowlist + k) : 0u;
            const float4 pi = __ldg(S.pos + ii);
            double sum = 0.0;
            for (uint32_t t = 0; t < T; t++) {
                const uint4 c = ld_mat(cols + 32 * t, pol);
                const float4 w = chunk_weights<EX, SW>(wts + 32 * t, pol, S.pos, S.rlap, S.rlap_thr, pi, ii, c);
                sum += (double)w.x * S.x64[c.x] + (double)w.y * S.x64[c.y] + (double)w.z * S.x64[c.z] +
                       (double)w.w * S.x64[c.w];
            }
            sum += __shfl_xor_sync(0xffffffffu, sum, 8);
            sum += __shfl_xor_sync(0xffffffffu, sum, 16);
            if (q == 0 && k < R) {
                const double bi = S.b64[ii];
                const double ri = bi - (S.diag64[ii] * S.x64[ii] + sum);
                const float rf = (float)ri;
                S.r[ii] = rf;
                S.u[ii] = rf * S.inv_diag[ii];
                acc[0] += ri * ri;
                acc[1] += bi * bi;
            }
        }
        double tot[2];
        if (!grid_reduce<2>(acc, S.part, S.result, S.bar, S.sc, tot)) return;
        outers++;
        const double rr64 = tot[0], bb = tot[1];
        relres = bb > 0.0 ? sqrt(rr64 / bb) : 0.0;
        if (relres <= S.tol) {
            converged = true;
            break;
        }
        if (total >= S.max_iter) break;
        // ---- w = A u, m = M w; gamma = r.u, delta = w.u; z = q = s = p = 0
        double g0[3] = {0.0, 0.0, 0.0};
        for (uint32_t sl = gw; sl < nslices; sl += nw) {
            const uint32_t k = sl * SELL_C + rsub;
            const uint32_t base = __ldg(S.off + sl);
            const uint64_t pol = mat_policy(base, S.keep);
            const uint32_t T = (__ldg(S.off + sl + 1) - base) >> 7;
            const uint4* cols = reinterpret_cast<const uint4*>(S.scols + base) + lane;
            const float4* wts = reinterpret_cast<const float4*>(S.sw + base) + lane;
            const uint32_t ii = k < R ? __ldg(rowlist + k) : 0u;
            const float4 pi = __ldg(S.pos + ii);
            float s0 = 0.f, s1 = 0.f;
            for (uint32_t t = 0; t < T; t++) {
                const uint4 c = ld_mat(cols + 32 * t, pol);
                const float4 w = chunk_weights<EX, SW>(wts + 32 * t, pol, S.pos, S.rlap, S.rlap_thr, pi, ii, c);
                s0 = fmaf(w.x, S.u[c.x], s0);
                s1 = fmaf(w.y, S.u[c.y], s1);
                s0 = fmaf(w.z, S.u[c.z], s0);
                s1 = fmaf(w.w, S.u[c.w], s1);
            }
            float sum = s0 + s1;
            sum += __shfl_xor_sync(0xffffffffu, sum, 8);
            sum += __shfl_xor_sync(0xffffffffu, sum, 16);
            if (q == 0 && k < R) {
                const float ui = S.u[ii];
                const float wi = fmaf(S.diag32[ii], ui, sum);
                S.w[ii] = wi;
                mc[ii] = wi * S.inv_diag[ii];
                S.z[ii] = 0.f;
                S.q[ii] = 0.f;
                S.s[ii] = 0.f;
                S.p[ii] = 0.f;
                const float ri = S.r[ii];
                g0[0] += (double)ri * (double)ui;
                g0[1] += (double)wi * (double)ui;
                g0[2] += (double)ri * (double)ri;
            }
        }
        double gt[3];
        if (!grid_reduce<3>(g0, S.part, S.result, S.bar, S.sc, gt)) return;
        double eta = 0.3 * S.tol / relres;
        if (eta < S.eta_min) eta = S.eta_min;
        if (eta > 0.5) eta = 0.5;
        const double stop = eta * eta * rr64;
        double gamma = gt[0], delta = gt[1], gamma_old = 1.0, alpha_old = 1.0;
        for (int it = 0; it < S.inner_cap && total < S.max_iter; it++) {
            double beta = 0.0, alpha;
            if (it == 0) {
                alpha = gamma / delta;
            } else {
                beta = gamma / gamma_old;
                alpha = gamma / (delta - beta * gamma / alpha_old);
            }
            const float bf = (float)beta, af = (float)alpha;
            // ---- n = A m; z, q, s, p, x, r, u, w updates; r.u, w.u, r.r
            double g[3] = {0.0, 0.0, 0.0};
            for (uint32_t sl = gw; sl < nslices; sl += nw) {
                const uint32_t k = sl * SELL_C + rsub;
                const uint32_t base = __ldg(S.off + sl);
                const uint64_t pol = mat_policy(base, S.keep);
                const uint32_t T = (__ldg(S.off + sl + 1) - base) >> 7;
                const uint4* cols = reinterpret_cast<const uint4*>(S.scols + base) + lane;
                const float4* wts = reinterpret_cast<const float4*>(S.sw + base) + lane;
                const uint32_t ii = k < R ? __ldg(rowlist + k) : 0u;
                const float4 pi = __ldg(S.pos + ii);
                float s0 = 0.f, s1 = 0.f;
#pragma unroll 4
                for (uint32_t t = 0; t < T; t++) {
                    const uint4 c = ld_mat(cols + 32 * t, pol);
                    const float4 w = chunk_weights<EX, SW>(wts + 32 * t, pol, S.pos, S.rlap, S.rlap_thr, pi, ii, c);
                    s0 = fmaf(w.x, mc[c.x], s0);
                    s1 = fmaf(w.y, mc[c.y], s1);
                    s0 = fmaf(w.z, mc[c.z], s0);
                    s1 = fmaf(w.w, mc[c.w], s1);
                }
                float sum = s0 + s1;
                sum += __shfl_xor_sync(0xffffffffu, sum, 8);
                sum += __shfl_xor_sync(0xffffffffu, sum, 16);
                if (q == 0 && k < R) {
                    const float mi = mc[ii];
                    const float ni = fmaf(S.diag32[ii], mi, sum);
                    const float zi = fmaf(bf, S.z[ii], ni);
                    const float qi = fmaf(bf, S.q[ii], mi);
                    const float wi0 = S.w[ii];
                    const float si = fmaf(bf, S.s[ii], wi0);
                    const float pin = fmaf(bf, S.p[ii], S.u[ii]);
                    S.x64[ii] += alpha * (double)pin;
                    const float ri = fmaf(-af, si, S.r[ii]);
                    const float ui = fmaf(-af, qi, S.u[ii]);
                    const float wi = fmaf(-af, zi, wi0);
                    S.z[ii] = zi;
                    S.q[ii] = qi;
                    S.s[ii] = si;
                    S.p[ii] = pin;
                    S.r[ii] = ri;
                    S.u[ii] = ui;
                    S.w[ii] = wi;
                    mn[ii] = wi * S.inv_diag[ii];
                    g[0] += (double)ri * (double)ui;
                    g[1] += (double)wi * (double)ui;
                    g[2] += (double)ri * (double)ri;
                }
            }
            double gg[3];
            if (!grid_reduce<3>(g, S.part, S.result, S.bar, S.sc, gg)) return;
            total++;
            gamma_old = gamma;
            alpha_old = alpha;
            gamma = gg[0];
            delta = gg[1];
            float* t = mc;
            mc = mn;
            mn = t;
            if (gg[2] <= stop) break;
        }
        // the last iteration ended on a grid-wide reduction, so every x64
        // update is visible to the residual pass of the next round
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        S.sc->cg_iters = total;
        S.sc->cg_outer = outers;
        S.sc->cg_relres = relres;
        if (!converged) atomicOr(&S.sc->err, ERR_CG_NOT_CONVERGED);
    }
}

// ---------------------------------------------------------------- batched solve
// The scenes of a batch in one persistent launch.  Each scene runs its own
// diagonally scaled PCG (its own alpha, beta, inner stop and FP64 true
// residual) exactly as a single scene does; the scenes share the grid
// barriers, and a scene that has met its inner target idles until the
// others reach theirs (or the inner cap), then every unconverged scene takes
// its next FP64 true-residual pass.  Per-scene sums are added in shared
// memory (a warp whose rows share one scene adds once), written per block,
// and the last block to arrive adds the blocks in order.
struct BatchSolveArgs {
    const uint32_t* rowlist;
    const uint32_t* nrows;
    const uint32_t* row_scene;
    const uint32_t* off;
    const uint32_t* scols;
    const float* sw;
    const float4* pos;
    const Phys* phys;
    const double* b64;
    const double* diag64;
    const float* diag32;
    const float* inv_diag;
    double* x64;
    float *r, *q;
    float2 *zp0, *zp1;
    double* part;
    double* result;
    unsigned* bar;
    Scalars* sc;
    int* iters;
    int* outers;
    double* relres;
    // learned preconditioner S' by particle columns (ppe_device.cuh) and its
    // (r, q) pair buffers, as in SolveArgs
    const uint32_t* sp_off;
    const uint32_t* sp_ent;
    const float* sp_diag;
    float2* rq0;
    float2* rq1;
    uint32_t ns;
    double tol;
    double eta_min;
    uint32_t keep;
    int max_iter, inner_cap, max_outer;
};

// add v[k] of every contributing lane to acc[k * ns + s] (whole warp calls)
template <int K>
__device__ __forceinline__ void scene_add(double* acc, uint32_t ns, uint32_t s, bool contrib, const double (&v)[K]) {
    const uint32_t s0 = __shfl_sync(0xffffffffu, s, 0);
    if (__all_sync(0xffffffffu, !contrib || s == s0)) {
#pragma unroll
        for (int k = 0; k < K; k++) {
            const double t = warp_sum_d(contrib ? v[k] : 0.0);
            if ((threadIdx.x & 31) == 0) atomicAdd(acc + k * ns + s0, t);
        }
    } else if (contrib) {
#pragma unroll
        for (int k = 0; k < K; k++) atomicAdd(acc + k * ns + s, v[k]);
    }
}

// Grid-wide per-scene sums (acc: this block's K * ns sums in shared memory,
// replaced by the totals) fused with a grid barrier; bounded wait as in
// grid_reduce.
template <int K>
__device__ bool grid_reduce_scenes(double* acc, uint32_t ns, double* part, double* result, unsigned* bar, Scalars* sc) {
    __syncthreads();
    const uint32_t m = K * ns;
    for (uint32_t t = threadIdx.x; t < m; t += blockDim.x) part[(size_t)blockIdx.x * m + t] = acc[t];
    __threadfence();
    __shared__ int last, ok;
    __shared__ unsigned gen0;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        volatile unsigned* gen = bar + 1;
        gen0 = *gen;
        __threadfence();
        last = atomicAdd(bar, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last) {
        // `per` threads share each of the m sums: thread g of a value adds
        // blocks g, g + per, ... (eight loads in flight), and the value's
        // first thread adds the per partial sums in order
        __shared__ double red[PPE_THREADS];
        __threadfence();
        const uint32_t per = blockDim.x >= m ? blockDim.x / m : 1u;
        const uint32_t vals = blockDim.x / per;
        const uint32_t G = gridDim.x;
        for (uint32_t v0 = 0; v0 < m; v0 += vals) {
            const uint32_t t = v0 + threadIdx.x / per, g = threadIdx.x % per;
            double sum = 0.0;
            if (threadIdx.x < vals * per && t < m) {
                for (uint32_t b = g; b < G; b += 8 * per) {
                    double v8[8];
#pragma unroll
                    for (int u = 0; u < 8; u++) {
                        const uint32_t bb = b + u * per;
                        v8[u] = bb < G ? __ldcg(part + (size_t)bb * m + t) : 0.0;
                    }
#pragma unroll
                    for (int u = 0; u < 8; u++) sum += v8[u];
                }
            }
            red[threadIdx.x] = sum;
            __syncthreads();
            if (g == 0 && threadIdx.x < vals * per && t < m) {
                double v = 0.0;
                for (uint32_t k = 0; k < per; k++) v += red[threadIdx.x + k];
                result[t] = v;
            }
            __syncthreads();
        }
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        }
    } else if (threadIdx.x == 0) {
        volatile unsigned* gen = bar + 1;
        const unsigned long long budget = wait_budget_ns(sc);
        uint64_t t0;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
        while (*gen == gen0) {
            uint64_t t1;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t1));
            if (t1 - t0 > budget) {
                atomicOr(&sc->err, ERR_DEVICE_TIMEOUT);
                ok = 0;
                break;
            }
            __nanosleep(32);
        }
        __threadfence();
    }
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < m; t += blockDim.x) acc[t] = __ldcg(result + t);
    const bool good = ok != 0;
    __syncthreads();
    return good;
}

template <bool EX>
__device__ __forceinline__ float batch_weight(const float4* __restrict__ pos, float rlap, float thr, const float4& pi,
                                              uint32_t i, uint32_t j) {
    const float4 pj = __ldg(pos + j);
    const float dx = fsub<EX>(pj.x, pi.x), dy = fsub<EX>(pj.y, pi.y), dz = fsub<EX>(pj.z, pi.z);
    const float rr = dot3<EX>(dx, dy, dz, dx, dy, dz);
    return (j != i && rr < thr) ? weight_rr<EX>(rlap, rr) : 0.f;
}

// PREC 0: diagonal scaling; PREC 1: the learned S' (neighbours of a row are
// rows of its own scene, so one pass of z = S' r serves all scenes still
// iterating; each neighbour's new residual is formed on the fly with its
// scene's alpha, the row's own goes to the second residual buffer).  Both
// keep two grid-wide reductions per iteration.  The residual buffers swap
// after every iteration; the rows of a scene that sits the iteration out
// keep theirs in the other buffer, which is harmless: a scene becomes active
// again only after the next FP64 pass, which rewrites the residual of every
// open scene's rows into the current buffer.
template <bool EX, bool SW, int PREC>
__global__ void __launch_bounds__(PPE_THREADS) k_ppe_solve_batch(BatchSolveArgs S) {
    __shared__ double acc[3 * PPE_MAX_SCENES];
    __shared__ double rz[PPE_MAX_SCENES], stop[PPE_MAX_SCENES], alpha[PPE_MAX_SCENES], rel[PPE_MAX_SCENES];
    __shared__ float beta[PPE_MAX_SCENES];
    __shared__ int its[PPE_MAX_SCENES], outs[PPE_MAX_SCENES];
    __shared__ unsigned char active[PPE_MAX_SCENES], done[PPE_MAX_SCENES];
    __shared__ int n_open, n_active;
    const uint32_t ns = S.ns;
    const uint32_t R = *S.nrows;
    const uint32_t nslices = (R + SELL_C - 1) / SELL_C;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t rsub = lane & 7, q = lane >> 3;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t* __restrict__ rowlist = S.rowlist;
    for (uint32_t s = threadIdx.x; s < ns; s += blockDim.x) {
        done[s] = 0;
        active[s] = 0;
        its[s] = 0;
        outs[s] = 0;
        rel[s] = 0.0;
    }
    int total = 0;
    float2* zc = S.zp0;   // (z, p) per row, current and next
    float2* zn = S.zp1;
    float2* rqc = S.rq0;  // learned: the (r, q) pairs, and the buffer its update writes
    float2* rqn = S.rq1;
    for (int outer = 0; outer < S.max_outer; outer++) {
        for (uint32_t t = threadIdx.x; t < 3 * ns; t += blockDim.x) acc[t] = 0.0;
        __syncthreads();
        // ---- FP64 true residual of the unconverged scenes' rows
        for (uint32_t sl = gw; sl < nslices; sl += nw) {
            const uint32_t k = sl * SELL_C + rsub;
            const bool has = k < R;
            const uint32_t ii = has ? __ldg(rowlist + k) : 0u;
            const uint32_t s = has ? __ldg(S.row_scene + k) : 0u;
            const bool work = has && !done[s];
            if (!__any_sync(0xffffffffu, work)) continue;
            const uint32_t base = __ldg(S.off + sl);
            const uint64_t pol = mat_policy(base, S.keep);
            const uint32_t T = (__ldg(S.off + sl + 1) - base) >> 7;
            const uint4* cols = reinterpret_cast<const uint4*>(S.scols + base) + lane;
            const float4* wts = reinterpret_cast<const float4*>(S.sw + base) + lane;
            const float4 pi = __ldg(S.pos + ii);
            const float rl = S.phys[s].rlap, thr = S.phys[s].rlap_thr;
            double sum = 0.0;
            if (work)
                for (uint32_t t = 0; t < T; t++) {
                    const uint4 c = ld_mat(cols + 32 * t, pol);
                    const float4 w = chunk_weights<EX, SW>(wts + 32 * t, pol, S.pos, rl, thr, pi, ii, c);
                    sum += (double)w.x * S.x64[c.x] + (double)w.y * S.x64[c.y] + (double)w.z * S.x64[c.z] +
                           (double)w.w * S.x64[c.w];
                }
            sum += __shfl_xor_sync(0xffffffffu, sum, 8);
            sum += __shfl_xor_sync(0xffffffffu, sum, 16);
            const bool contrib = q == 0 && work;
            double v[3] = {0.0, 0.0, 0.0};
            if (contrib) {
                const double bi = S.b64[ii];
                const double ri = bi - (S.diag64[ii] * S.x64[ii] + sum);
                const float rf = (float)ri;
                const float zf = PREC == 0 ? rf * S.inv_diag[ii] : 0.f;
                if (PREC == 1) rqc[ii].x = rf;
                else S.r[ii] = rf;
                zc[ii] = make_float2(zf, 0.f);
                v[0] = ri * ri;
                v[1] = bi * bi;
                v[2] = (double)rf * (double)zf;
            }
            scene_add<3>(acc, ns, s, contrib, v);
        }
        if (!grid_reduce_scenes<3>(acc, ns, S.part, S.result, S.bar, S.sc)) return;
        for (uint32_t s = threadIdx.x; s < ns; s += blockDim.x) {
            if (done[s]) continue;
            const double rr64 = acc[s], bb = acc[ns + s];
            const double relres = bb > 0.0 ? sqrt(rr64 / bb) : 0.0;
            rel[s] = relres;
            outs[s]++;
            if (relres <= S.tol) {
                done[s] = 1;
                active[s] = 0;
            } else {
                double eta = 0.3 * S.tol / relres;
                if (eta < S.eta_min) eta = S.eta_min;
                if (eta > 0.5) eta = 0.5;
                active[s] = 1;
                rz[s] = acc[2 * ns + s];
                stop[s] = eta * eta * rr64;
                beta[s] = 0.f;
            }
        }
        __syncthreads();
        if (PREC == 1) {
            // z = S' r on the rows of the scenes still open; r.z per scene
            for (uint32_t t = threadIdx.x; t < ns; t += blockDim.x) acc[t] = 0.0;
            __syncthreads();
            for (uint32_t k0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); k0 < R; k0 += stride) {
                const uint32_t kk = k0 + lane;
                const bool has = kk < R;
                const uint32_t s = has ? __ldg(S.row_scene + kk) : 0u;
                const bool contrib = has && !done[s];
                double v[1] = {0.0};
                if (contrib) {
                    const uint32_t i = __ldg(rowlist + kk);
                    const float2* rq = rqc;
                    const float zi =
                        sp_row_at(S.sp_off, S.sp_ent, S.sp_diag, kk, i, [rq](uint32_t j) { return rq[j].x; });
                    zc[i].x = zi;
                    v[0] = (double)rq[i].x * (double)zi;
                }
                scene_add<1>(acc, ns, s, contrib, v);
            }
            if (!grid_reduce_scenes<1>(acc, ns, S.part, S.result, S.bar, S.sc)) return;
            for (uint32_t s = threadIdx.x; s < ns; s += blockDim.x)
                if (active[s]) rz[s] = acc[s];
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            int c = 0;
            for (uint32_t s = 0; s < ns; s++) c += done[s] ? 0 : 1;
            n_open = c;
        }
        __syncthreads();
        if (n_open == 0 || total >= S.max_iter) break;
        for (int it = 0; it < S.inner_cap && total < S.max_iter; it++) {
            for (uint32_t t = threadIdx.x; t < ns; t += blockDim.x) acc[t] = 0.0;
            __syncthreads();
            // ---- q = A p_new with p_new = z + beta p (fused), p.q per scene
            for (uint32_t sl = gw; sl < nslices; sl += nw) {
                const uint32_t k = sl * SELL_C + rsub;
                const bool has = k < R;
                const uint32_t ii = has ? __ldg(rowlist + k) : 0u;
                const uint32_t s = has ? __ldg(S.row_scene + k) : 0u;
                const bool work = has && active[s];
                if (!__any_sync(0xffffffffu, work)) continue;
                const uint32_t base = __ldg(S.off + sl);
                const uint64_t pol = mat_policy(base, S.keep);
                const uint32_t T = (__ldg(S.off + sl + 1) - base) >> 7;
                const uint4* cols = reinterpret_cast<const uint4*>(S.scols + base) + lane;
                const float4* wts = reinterpret_cast<const float4*>(S.sw + base) + lane;
                const float4 pi = __ldg(S.pos + ii);
                const float rl = S.phys[s].rlap, thr = S.phys[s].rlap_thr;
                const float bs = beta[s];
                float sum = 0.f, sum1 = 0.f;
                if (work)
                    for (uint32_t t = 0; t < T; t++) {
                        const uint4 c = ld_mat(cols + 32 * t, pol);
                        const float4 w = chunk_weights<EX, SW>(wts + 32 * t, pol, S.pos, rl, thr, pi, ii, c);
                        const float2 a0 = zc[c.x], a1 = zc[c.y], a2 = zc[c.z], a3 = zc[c.w];
                        sum = fmaf(w.x, fmaf(bs, a0.y, a0.x), sum);
                        sum1 = fmaf(w.y, fmaf(bs, a1.y, a1.x), sum1);
                        sum = fmaf(w.z, fmaf(bs, a2.y, a2.x), sum);
                        sum1 = fmaf(w.w, fmaf(bs, a3.y, a3.x), sum1);
                    }
                sum += sum1;
                sum += __shfl_xor_sync(0xffffffffu, sum, 8);
                sum += __shfl_xor_sync(0xffffffffu, sum, 16);
                const bool contrib = q == 0 && work;
                double v[1] = {0.0};
                if (contrib) {
                    const float2 o = zc[ii];
                    const float pn = fmaf(bs, o.y, o.x);
                    const float qi = fmaf(S.diag32[ii], pn, sum);
                    zn[ii].y = pn;
                    if (PREC == 1) rqc[ii].y = qi;
                    else S.q[ii] = qi;
                    v[0] = (double)pn * (double)qi;
                }
                scene_add<1>(acc, ns, s, contrib, v);
            }
            if (!grid_reduce_scenes<1>(acc, ns, S.part, S.result, S.bar, S.sc)) return;
            for (uint32_t s = threadIdx.x; s < ns; s += blockDim.x)
                if (active[s]) alpha[s] = rz[s] / acc[s];
            __syncthreads();
            for (uint32_t t = threadIdx.x; t < 2 * ns; t += blockDim.x) acc[t] = 0.0;
            __syncthreads();
            // ---- x64 += alpha p, r -= alpha q, z = M^-1 r; r.z and r.r per scene
            if (PREC == 0) {
                for (uint32_t k0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); k0 < R; k0 += stride) {
                    const uint32_t kk = k0 + lane;
                    const bool has = kk < R;
                    const uint32_t s = has ? __ldg(S.row_scene + kk) : 0u;
                    const bool contrib = has && active[s];
                    double v[2] = {0.0, 0.0};
                    if (contrib) {
                        const uint32_t i = __ldg(rowlist + kk);
                        const double al = alpha[s];
                        const float pn = zn[i].y;
                        S.x64[i] += al * (double)pn;
                        const float ri = fmaf(-(float)al, S.q[i], S.r[i]);
                        const float zi = ri * S.inv_diag[i];
                        S.r[i] = ri;
                        zn[i] = make_float2(zi, pn);
                        v[0] = (double)ri * (double)zi;
                        v[1] = (double)ri * (double)ri;
                    }
                    scene_add<2>(acc, ns, s, contrib, v);
                }
                if (!grid_reduce_scenes<2>(acc, ns, S.part, S.result, S.bar, S.sc)) return;
            } else {
                // x64 += alpha p; z = S' r_new with each neighbour's r_new =
                // r - alpha q formed on the fly (same scene, same alpha); the
                // new residual into the other buffer; r.z and r.r per scene
                for (uint32_t k0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); k0 < R; k0 += stride) {
                    const uint32_t kk = k0 + lane;
                    const bool has = kk < R;
                    const uint32_t s = has ? __ldg(S.row_scene + kk) : 0u;
                    const bool contrib = has && active[s];
                    double v[2] = {0.0, 0.0};
                    if (contrib) {
                        const uint32_t i = __ldg(rowlist + kk);
                        const double al = alpha[s];
                        const float af = (float)al;
                        const float pn = zn[i].y;
                        S.x64[i] += al * (double)pn;
                        const float2* rq = rqc;
                        const float2 o = rq[i];
                        const float ri = fmaf(-af, o.y, o.x);
                        rqn[i] = make_float2(ri, 0.f);
                        const float zi = sp_row_at(S.sp_off, S.sp_ent, S.sp_diag, kk, i, [rq, af](uint32_t j) {
                            const float2 v = rq[j];
                            return fmaf(-af, v.y, v.x);
                        });
                        zn[i] = make_float2(zi, pn);
                        v[0] = (double)ri * (double)zi;
                        v[1] = (double)ri * (double)ri;
                    }
                    scene_add<2>(acc, ns, s, contrib, v);
                }
                if (!grid_reduce_scenes<2>(acc, ns, S.part, S.result, S.bar, S.sc)) return;
                float2* t_ = rqc;
                rqc = rqn;
                rqn = t_;
            }
            for (uint32_t s = threadIdx.x; s < ns; s += blockDim.x) {
                if (!active[s]) continue;
                beta[s] = (float)(acc[s] / rz[s]);
                rz[s] = acc[s];
                its[s]++;
                if (acc[ns + s] <= stop[s]) active[s] = 0;
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                int c = 0;
                for (uint32_t s = 0; s < ns; s++) c += active[s] ? 1 : 0;
                n_active = c;
            }
            __syncthreads();
            total++;
            float2* t = zc;
            zc = zn;
            zn = t;
            if (n_active == 0) break;
        }
    }
    if (blockIdx.x == 0) {
        for (uint32_t s = threadIdx.x; s < ns; s += blockDim.x) {
            S.iters[s] = its[s];
            S.outers[s] = outs[s];
            S.relres[s] = rel[s];
            if (!done[s]) atomicOr(&S.sc->err, ERR_CG_NOT_CONVERGED);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int mi = 0, mo = 0;
            double mr = 0.0;
            for (uint32_t s = 0; s < ns; s++) {
                mi = its[s] > mi ? its[s] : mi;
                mo = outs[s] > mo ? outs[s] : mo;
                mr = rel[s] > mr ? rel[s] : mr;
            }
            S.sc->cg_iters = mi;
            S.sc->cg_outer = mo;
            S.sc->cg_relres = mr;
        }
    }
}

// scene of every row (batch)
__global__ void __launch_bounds__(256) k_row_scene(const uint32_t* __restrict__ rowlist, const uint32_t* __restrict__ nrows,
                                                   const uint32_t* __restrict__ id, const uint32_t* __restrict__ sid_of_id,
                                                   uint32_t* __restrict__ row_scene, uint32_t cap) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= *nrows || k >= cap) return;
    row_scene[k] = sid_of_id[id[rowlist[k]]];
}

// ---------------------------------------------------------------- row list
// Ordered list of the non-Dirichlet rows: the solver splits it into equal
// contiguous slices per block (Dirichlet and dummy rows cluster in space, so
// slicing the particle range would leave some blocks idle).
constexpr uint32_t ROW_TILE = 2048;

__global__ void __launch_bounds__(256) k_rows_count(const uint32_t* __restrict__ rlen, const Scalars* __restrict__ sc,
                                                    uint32_t* __restrict__ tilecnt) {
    const uint32_t n = sc->np;
    const uint32_t base = blockIdx.x * ROW_TILE;
    uint32_t c = 0;
    for (uint32_t k = threadIdx.x; k < ROW_TILE; k += blockDim.x) {
        const uint32_t i = base + k;
        if (i < n && rlen[i] != PPE_DIRICHLET) c++;
    }
    c = __reduce_add_sync(0xffffffffu, c);
    __shared__ uint32_t ws[8];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < 8; w++) t += ws[w];
        tilecnt[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(256) k_rows_scatter(const uint32_t* __restrict__ rlen, const Scalars* __restrict__ sc,
                                                      const uint32_t* __restrict__ tileoff, uint32_t ntiles,
                                                      uint32_t* __restrict__ rowlist, uint32_t* __restrict__ nrows) {
    const uint32_t n = sc->np;
    const uint32_t base = blockIdx.x * ROW_TILE;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __shared__ uint32_t ws[8];
    __shared__ uint32_t run;
    if (threadIdx.x == 0) run = tileoff[blockIdx.x];
    __syncthreads();
    for (uint32_t k0 = 0; k0 < ROW_TILE; k0 += blockDim.x) {
        const uint32_t i = base + k0 + threadIdx.x;
        const bool f = i < n && rlen[i] != PPE_DIRICHLET;
        const uint32_t m = __ballot_sync(0xffffffffu, f);
        if (lane == 0) ws[warp] = __popc(m);
        __syncthreads();
        uint32_t off = run;
        for (uint32_t w = 0; w < warp; w++) off += ws[w];
        if (f) rowlist[off + __popc(m & ((1u << lane) - 1u))] = i;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t t = 0;
            for (int w = 0; w < 8; w++) t += ws[w];
            run += t;
        }
        __syncthreads();
    }
    if (blockIdx.x == ntiles - 1 && threadIdx.x == 0) *nrows = run;
}

// ---------------------------------------------------------------- SELL-8
// Sliced ELL: slice s holds rows rowlist[8s .. 8s+7], width W_s = the
// longest of them rounded up to a multiple of 16, padded with the row's own
// index and weight 0.  A warp takes one slice with 4 lanes per row; lane
// L = 8q + r owns, in every chunk t of 16 entries of row r, the 4 entries
// 16t + q, 16t + q + 4, 16t + q + 8 and 16t + q + 12, stored together at word
// sell_off[s] + 4 (32t + L), so each lane reads them (columns, and weights
// in the same layout) as one 16-byte vector and a warp's load is one
// contiguous 512-byte block; the four lanes of a row then gather four
// consecutive entries per instruction.
__global__ void __launch_bounds__(256) k_sell_width(const uint32_t* __restrict__ rlen,
                                                    const uint32_t* __restrict__ rowlist,
                                                    const uint32_t* __restrict__ nrows, uint32_t* __restrict__ width,
                                                    uint32_t maxslices) {
    const uint32_t R = *nrows;
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;  // slice
    if (s > maxslices) return;
    uint32_t m = 0;
    const uint32_t k0 = s * SELL_C;
    for (uint32_t r = 0; r < SELL_C; r++) {
        const uint32_t k = k0 + r;
        if (k < R) m = max(m, rlen[rowlist[k]]);
    }
    width[s] = SELL_C * ((m + 15u) & ~15u);
}

// Columns and weights of the assembly, repacked (padding: the row's own
// index, weight 0).  One warp per slice: in chunk t, lane L = r + 8q moves
// the 4 entries 16t + 4q .. 16t + 4q + 3 of row r as one 16-byte load from
// the row-major scratch and one 16-byte store, so the warp writes its 512
// bytes contiguously.
__global__ void __launch_bounds__(256) k_sell_pack(const uint32_t* __restrict__ cols_rm, const float* __restrict__ w_rm,
                                                   const uint32_t* __restrict__ rlen, const uint32_t* __restrict__ rowlist,
                                                   const uint32_t* __restrict__ nrows, const uint32_t* __restrict__ off,
                                                   uint32_t* __restrict__ scols, float* __restrict__ sw) {
    const uint32_t R = *nrows;
    const uint32_t slice = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31, r = lane & 7, q = lane >> 3;
    if (slice >= (R + SELL_C - 1) / SELL_C) return;
    const uint32_t base = off[slice];
    const uint32_t T = (off[slice + 1] - base) >> 7;  // chunks of 16 entries per row
    const uint32_t k = slice * SELL_C + r;
    const bool has = k < R;
    const uint32_t i = has ? rowlist[k] : 0u;
    const uint32_t len = has ? rlen[i] : 0u;
    const uint32_t* rc = cols_rm + (size_t)i * PPE_W;
    const float* rw = w_rm + (size_t)i * PPE_W;
    uint4* dc = reinterpret_cast<uint4*>(scols + base) + lane;
    float4* dw = reinterpret_cast<float4*>(sw + base) + lane;
    for (uint32_t t = 0; t < T; t++) {
        // lane (r, q) holds entries q, q + 4, q + 8, q + 12 of the row's 16
        // in this chunk, so that one gather instruction of the solver reads
        // 4 consecutive entries of each row: neighbouring columns, mostly in
        // the same 32-byte sectors of the gathered vector
        const uint32_t e = 16u * t + q;
        uint4 c = make_uint4(i, i, i, i);
        float4 w = make_float4(0.f, 0.f, 0.f, 0.f);
        if (e < len) { c.x = rc[e]; w.x = rw[e]; }
        if (e + 4 < len) { c.y = rc[e + 4]; w.y = rw[e + 4]; }
        if (e + 8 < len) { c.z = rc[e + 8]; w.z = rw[e + 8]; }
        if (e + 12 < len) { c.w = rc[e + 12]; w.w = rw[e + 12]; }
        dc[32 * t] = c;
        dw[32 * t] = w;
    }
}

// p = max(x, 0) (pressCorr, MPS_CAL_v4.0/MPS_CPU.cpp:734-743); Dirichlet rows 0.
__global__ void __launch_bounds__(256) k_ppe_finish(const double* __restrict__ x64, const uint32_t* __restrict__ rlen,
                                                    float* __restrict__ press, const Scalars* __restrict__ sc) {
    const uint32_t n = sc->np;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float p = 0.f;
    if (rlen[i] != PPE_DIRICHLET) {
        p = (float)x64[i];
        if (p < 0.f) p = 0.f;
    }
    press[i] = p;
}

// ---------------------------------------------------------------- FP64 init
// n of every particle in double (weights from the float positions in double)
__global__ void __launch_bounds__(256) k_pnd64(StageArgs a, double* __restrict__ n64) {
    const uint32_t n = a.sc->np;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4* __restrict__ pos = a.cur.pos;
    const float4 pi = pos[i];
    const Local L = local_of(a, i);
    const double re = (double)phys_of(a, L.s).rzero;
    double acc = 0.0;
    const int rows = link_rows(L.g);
    for (int row = 0; row < rows; row++) {
        const RowRange rg = link_row(L.g, L.cs, L.c, row);
        for (uint32_t j = rg.lo; j < rg.hi; j++) {
            if (j == i) continue;
            const float4 pj = __ldg(pos + j);
            const double dx = (double)pj.x - pi.x, dy = (double)pj.y - pi.y, dz = (double)pj.z - pi.z;
            const double r = sqrt(dx * dx + dy * dy + dz * dz);
            if (r < re) acc += re / r - 1.0;
        }
    }
    n64[i] = acc;
    a.cur.n[i] = (float)acc;
}

void launch_pnd64(const StageArgs& a, double* n64, uint32_t cap, cudaStream_t st) {
    k_pnd64<<<blocks_for(cap, 256), 256, 0, st>>>(a, n64);
}

// n0 = the first maximum of n in GEO.dat order (the reference's calOnce
// runs before the first sort, MPS_CAL_v4.0/MPS.cpp:316-333): the largest n64,
// smallest id on ties; then lambda = sum r^2 w(r; r0) / n0 around it
// (MPS.cpp:335-348).  One block.
__global__ void __launch_bounds__(1024) k_n0_lambda64(StageArgs a, const double* __restrict__ n64, double* out,
                                                     uint32_t lo, uint32_t hi) {
    __shared__ double sn[1024];
    __shared__ uint32_t sid[1024], sidx[1024];
    const uint32_t np = hi < a.sc->np ? hi : a.sc->np;
    double bn = -1.0;
    uint32_t bid = 0xffffffffu, bix = 0xffffffffu;
    for (uint32_t i = lo + threadIdx.x; i < np; i += blockDim.x) {
        const double v = n64[i];
        const uint32_t id = a.cur.id[i];
        if (v > bn || (v == bn && id < bid)) { bn = v; bid = id; bix = i; }
    }
    sn[threadIdx.x] = bn; sid[threadIdx.x] = bid; sidx[threadIdx.x] = bix;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            const double v = sn[threadIdx.x + o];
            const uint32_t id = sid[threadIdx.x + o];
            if (v > sn[threadIdx.x] || (v == sn[threadIdx.x] && id < sid[threadIdx.x])) {
                sn[threadIdx.x] = v; sid[threadIdx.x] = id; sidx[threadIdx.x] = sidx[threadIdx.x + o];
            }
        }
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    const uint32_t t = sidx[0];
    const double n0 = sn[0];
    if (t == 0xffffffffu || !(n0 > 0.0)) { out[0] = 0.0; out[1] = 0.0; return; }
    const float4 pt = a.cur.pos[t];
    const Local L = local_of(a, t);
    const double re = (double)phys_of(a, L.s).rzero;
    double lam = 0.0;
    const int rows = link_rows(L.g);
    for (int row = 0; row < rows; row++) {
        const RowRange rg = link_row(L.g, L.cs, L.c, row);
        for (uint32_t j = rg.lo; j < rg.hi; j++) {
            if (j == t) continue;
            const float4 pj = a.cur.pos[j];
            const double dx = (double)pj.x - pt.x, dy = (double)pj.y - pt.y, dz = (double)pj.z - pt.z;
            const double r = sqrt(dx * dx + dy * dy + dz * dz);
            if (r < re) lam += r * r * (re / r - 1.0);
        }
    }
    out[0] = n0;
    out[1] = lam / n0;
}

void launch_n0_lambda64(const StageArgs& a, const double* n64, double* out, cudaStream_t st, uint32_t lo,
                        uint32_t hi) {
    k_n0_lambda64<<<1, 1024, 0, st>>>(a, n64, out, lo, hi);
}

// ---------------------------------------------------------------- host side
// every variant of the persistent solver (cooperative launches must fit)
static std::vector<const void*> solve_kernels() {
    return {(const void*)k_ppe_solve<true, 0, true>,    (const void*)k_ppe_solve<false, 0, true>,
            (const void*)k_ppe_solve<true, 1, true>,    (const void*)k_ppe_solve<false, 1, true>,
            (const void*)k_ppe_solve<true, 0, false>,   (const void*)k_ppe_solve<false, 0, false>,
            (const void*)k_ppe_solve<true, 1, false>,   (const void*)k_ppe_solve<false, 1, false>,
            (const void*)k_ppe_solve_batch<true, true, 0>, (const void*)k_ppe_solve_batch<false, true, 0>,
            (const void*)k_ppe_solve_batch<true, false, 0>, (const void*)k_ppe_solve_batch<false, false, 0>,
            (const void*)k_ppe_solve_batch<true, true, 1>, (const void*)k_ppe_solve_batch<false, true, 1>,
            (const void*)k_ppe_solve_batch<true, false, 1>, (const void*)k_ppe_solve_batch<false, false, 1>,
            (const void*)k_ppe_solve_pipe<true, true>,  (const void*)k_ppe_solve_pipe<false, true>,
            (const void*)k_ppe_solve_pipe<true, false>, (const void*)k_ppe_solve_pipe<false, false>};
}

int ppe_setup(PpeWork& w, uint32_t cap, const Grid&, const Phys&, const mps_params& prm, cudaStream_t st,
              std::string* err) {
    w.cap = cap;
    w.alpha64 = 1.0 / ((double)prm.rho * (double)prm.cs * (double)prm.cs);
    auto al = [&](void** p, size_t bytes) -> bool {
        if (cudaMalloc(p, bytes + 64) != cudaSuccess) return false;
        cudaMemsetAsync(*p, 0, bytes + 64, st);
        return true;
    };
    bool ok = true;
    ok &= al((void**)&w.cols, (size_t)cap * PPE_W * sizeof(uint32_t));
    ok &= al((void**)&w.wrm, (size_t)cap * PPE_W * sizeof(float));
    ok &= al((void**)&w.rlen, (size_t)cap * sizeof(uint32_t));
    ok &= al((void**)&w.diag64, (size_t)cap * sizeof(double));
    ok &= al((void**)&w.diag32, (size_t)cap * sizeof(float));
    ok &= al((void**)&w.inv_diag, (size_t)cap * sizeof(float));
    ok &= al((void**)&w.b64, (size_t)cap * sizeof(double));
    ok &= al((void**)&w.x64, (size_t)cap * sizeof(double));
    ok &= al((void**)&w.r, (size_t)cap * sizeof(float));
    for (float** v : {&w.pu, &w.pw, &w.pz, &w.pq, &w.ps, &w.pp, &w.pm[0], &w.pm[1]})
        ok &= al((void**)v, (size_t)cap * sizeof(float));
    ok &= al((void**)&w.zp[0], (size_t)cap * sizeof(float2));
    ok &= al((void**)&w.zp[1], (size_t)cap * sizeof(float2));
    ok &= al((void**)&w.q, (size_t)cap * sizeof(float));
    ok &= al((void**)&w.qp, (size_t)cap * (PPE_MAX_SPLIT - 1) * sizeof(float));
    ok &= al((void**)&w.rowlist, (size_t)cap * sizeof(uint32_t));
    ok &= al((void**)&w.pos_snap, (size_t)cap * sizeof(float4));
    ok &= al((void**)&w.n_snap, (size_t)cap * sizeof(float));
    ok &= al((void**)&w.id_snap, (size_t)cap * sizeof(uint32_t));
    ok &= al((void**)&w.sell_off, ((size_t)cap / SELL_C + 4) * sizeof(uint32_t));
    ok &= al((void**)&w.sell_cols, ((size_t)cap + 8) * (PPE_W + 4) * sizeof(uint32_t));
    ok &= al((void**)&w.sell_w, ((size_t)cap + 8) * (PPE_W + 4) * sizeof(float));
    ok &= al((void**)&w.tilecnt, ((size_t)cap / 2048 + 2) * sizeof(uint32_t));
    ok &= al((void**)&w.nrows, sizeof(uint32_t));
    if (!ok) {
        *err = "cudaMalloc failed for the PPE matrix";
        return MPS_ERR_CUDA;
    }
    int dev = 0, sms = 0, per_sm = 0, coop = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    {
        per_sm = 1 << 30;
        for (const void* f : solve_kernels()) {
            int o = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, f, PPE_THREADS, 0);
            per_sm = o < per_sm ? o : per_sm;
        }
    }
    if (!coop || per_sm < 1) {
        *err = "device cannot run the cooperative PPE solver";
        return MPS_ERR_CUDA;
    }
    if (per_sm > 1) per_sm = 1;
    {
        const int most = PPE_THREADS / 32 * PPE_SMEM_CHUNKS * 32 * (int)(sizeof(uint4) + sizeof(float4));
        for (const void* f : {(const void*)k_ppe_solve<true, 0, true>, (const void*)k_ppe_solve<false, 0, true>,
                              (const void*)k_ppe_solve<true, 1, true>, (const void*)k_ppe_solve<false, 1, true>})
            if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, most) != cudaSuccess) {
                *err = "the PPE solver cannot have its shared memory";
                return MPS_ERR_CUDA;
            }
    }
    w.sms = sms;
    w.threads = PPE_THREADS;
    w.blocks = sms * per_sm;
    // partials sized for the smallest block shape (4 blocks per SM)
    ok &= al((void**)&w.part, (size_t)sms * 4 * 2 * PPE_PARTS * sizeof(double));  // two buffers (grid_reduce)
    ok &= al((void**)&w.result, PPE_PARTS * sizeof(double));
    ok &= al((void**)&w.bar, 2 * sizeof(unsigned));
    if (!ok) {
        *err = "cudaMalloc failed for the PPE scratch";
        return MPS_ERR_CUDA;
    }
    w.ready = true;
    return MPS_OK;
}

// A cooperative launch through the launch-attribute form, which stream
// capture records as a cooperative graph kernel node.
static cudaError_t launch_cooperative(const void* fn, int blocks, int threads, void** args, cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)blocks);
    cfg.blockDim = dim3((unsigned)threads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelExC(&cfg, fn, args);
}

// The ordered list of non-Dirichlet rows and their SELL-8 layout (with the
// stored weights), from the assembled row-major system.
static int enqueue_rows_pack(PpeWork& w, const StageArgs& a, uint32_t cap, cudaStream_t st) {
    const uint32_t ntiles = (cap + ROW_TILE - 1) / ROW_TILE;
    k_rows_count<<<ntiles, 256, 0, st>>>(w.rlen, a.sc, w.tilecnt);
    launch_scan_exclusive(w.tilecnt, ntiles, st);
    k_rows_scatter<<<ntiles, 256, 0, st>>>(w.rlen, a.sc, w.tilecnt, ntiles, w.rowlist, w.nrows);
    int launched = 6;
    if (a.batch.n) {
        k_row_scene<<<blocks_for(cap, 256), 256, 0, st>>>(w.rowlist, w.nrows, a.cur.id, a.batch.sid_of_id, w.row_scene,
                                                          cap);
        launched++;
    }
    if (w.c16 && !a.batch.n) return launched + ppe_c16_enqueue_pack(w, a, cap, st);
    // SELL-8 layout of the non-Dirichlet rows
    const uint32_t maxslices = (cap + SELL_C - 1) / SELL_C;
    k_sell_width<<<blocks_for(maxslices + 1, 256), 256, 0, st>>>(w.rlen, w.rowlist, w.nrows, w.sell_off, maxslices);
    launch_scan_exclusive(w.sell_off, maxslices + 1, st);
    k_sell_pack<<<blocks_for(maxslices * 32u, 256), 256, 0, st>>>(w.cols, w.wrm, w.rlen, w.rowlist, w.nrows,
                                                                  w.sell_off, w.sell_cols, w.sell_w);
    return launched;
}

// The stored off-diagonal entries of every row, copied out of the solver's
// sliced layout into per-row lists (row i's entries at row_start[i] ..):
// the operator exactly as the solver reads it, for tests.
__global__ void __launch_bounds__(256) k_sell_export(const uint32_t* __restrict__ rlen,
                                                     const uint32_t* __restrict__ rowlist,
                                                     const uint32_t* __restrict__ nrows, const uint32_t* __restrict__ off,
                                                     const uint32_t* __restrict__ scols, const float* __restrict__ sw,
                                                     const uint32_t* __restrict__ row_start, uint32_t* __restrict__ cols,
                                                     float* __restrict__ wts) {
    const uint32_t R = *nrows;
    const uint32_t slice = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31, r = lane & 7, q = lane >> 3;
    if (slice >= (R + SELL_C - 1) / SELL_C) return;
    const uint32_t k = slice * SELL_C + r;
    if (k >= R) return;
    const uint32_t base = off[slice];
    const uint32_t T = (off[slice + 1] - base) >> 7;
    const uint32_t i = rowlist[k];
    const uint32_t len = rlen[i];
    const uint32_t o = row_start[i];
    for (uint32_t t = 0; t < T; t++) {
        for (uint32_t u = 0; u < 4; u++) {
            const uint32_t e = 16u * t + q + 4u * u;  // the pack's order (k_sell_pack)
            if (e < len) {
                const size_t src = (size_t)base + 4u * (32u * t + lane) + u;
                cols[o + e] = scols[src];
                wts[o + e] = sw[src];
            }
        }
    }
}

int ppe_export_stencil(const PpeWork& w, uint32_t np, uint32_t* row_start, uint32_t* cols, float* wts,
                       uint64_t max_entries, uint64_t* nnz, cudaStream_t st) {
    std::vector<uint32_t> len(np);
    if (np && cudaMemcpyAsync(len.data(), w.rlen, (size_t)np * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return MPS_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return MPS_ERR_CUDA;
    std::vector<uint32_t> start(np + 1);
    uint64_t t = 0;
    for (uint32_t i = 0; i < np; i++) {
        start[i] = (uint32_t)t;
        if (len[i] != PPE_DIRICHLET) t += len[i];
    }
    start[np] = (uint32_t)t;
    if (t > 0xffffffffull) return MPS_ERR_CAPACITY;
    if (nnz) *nnz = t;
    if (row_start) memcpy(row_start, start.data(), (size_t)(np + 1) * 4);
    if (!cols && !wts) return MPS_OK;
    if (t > max_entries) return MPS_ERR_CAPACITY;
    uint32_t *d_start = nullptr, *d_cols = nullptr;
    float* d_w = nullptr;
    int rc = MPS_OK;
    if (cudaMalloc(&d_start, (size_t)(np + 1) * 4) != cudaSuccess || cudaMalloc(&d_cols, (t + 1) * 4) != cudaSuccess ||
        cudaMalloc(&d_w, (t + 1) * 4) != cudaSuccess) {
        rc = MPS_ERR_CUDA;
    } else {
        cudaMemcpyAsync(d_start, start.data(), (size_t)(np + 1) * 4, cudaMemcpyHostToDevice, st);
        const uint32_t maxslices = (np + SELL_C - 1) / SELL_C;
        if (w.c16)
            ppe_c16_export(w, np, d_start, d_cols, d_w, st);
        else if (maxslices)
            k_sell_export<<<blocks_for(maxslices * 32u, 256), 256, 0, st>>>(w.rlen, w.rowlist, w.nrows, w.sell_off,
                                                                            w.sell_cols, w.sell_w, d_start, d_cols, d_w);
        if (cols) cudaMemcpyAsync(cols, d_cols, t * 4, cudaMemcpyDeviceToHost, st);
        if (wts) cudaMemcpyAsync(wts, d_w, t * 4, cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) rc = MPS_ERR_CUDA;
    }
    cudaFree(d_start);
    cudaFree(d_cols);
    cudaFree(d_w);
    return rc;
}

int ppe_enqueue_setup(PpeWork& w, const StageArgs& a, const mps_options& opt, uint32_t cap, cudaStream_t st) {
    (void)opt;
    AsmArgs A;
    A.a = a;
    A.cols = w.cols;
    A.wrm = w.wrm;
    A.rlen = w.rlen;
    A.diag64 = w.diag64;
    A.diag32 = w.diag32;
    A.inv_diag = w.inv_diag;
    A.b64 = w.b64;
    A.x64 = w.x64;
    A.bar = w.bar;
    A.n0 = w.n0_64;
    A.lambda = w.lambda64;
    A.beta = (double)a.P.beta;
    const double rho = (double)a.P.rho, dim = (double)a.P.dim_f;
    const double alpha = w.alpha64;
    const double one_over_dt = 1.0 / (double)a.P.dt_max;
    A.b_tmp = w.lambda64 * rho * (0.5 * (1.0 / dim) * one_over_dt * one_over_dt);
    A.rho_lambda_alpha_n0 = rho * w.lambda64 * alpha * w.n0_64;
    A.dim2 = 2.0 * dim;
    A.scenes = w.scenes;
    const uint32_t warps_blocks = blocks_for(cap * 32u, 256);
    if (a.batch.n) {
        if (a.exact) k_ppe_assemble<true, true><<<warps_blocks, 256, 0, st>>>(A);
        else k_ppe_assemble<false, true><<<warps_blocks, 256, 0, st>>>(A);
    } else {
        if (a.exact) k_ppe_assemble<true, false><<<warps_blocks, 256, 0, st>>>(A);
        else k_ppe_assemble<false, false><<<warps_blocks, 256, 0, st>>>(A);
    }
    int launched = 1 + enqueue_rows_pack(w, a, cap, st);
    // the state this system was assembled from
    cudaMemcpyAsync(w.pos_snap, a.cur.pos, (size_t)cap * sizeof(float4), cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(w.n_snap, a.cur.n, (size_t)cap * sizeof(float), cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(w.id_snap, a.cur.id, (size_t)cap * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st);
    w.have_snapshot = true;
    if (opt.precond == MPS_PRECOND_LEARNED && w.lp.ready && w.sp_ent) {
        // the symmetric form by GEO index, rebuilt every precond_every steps;
        // S' of the current rows every step (compact or particle columns)
        if (w.build_net) {
            const LpSystem L = ppe_lp_system(w, a);
            lp_build_stencil(w.lp, L, cap, st);
            lp_forward(w.lp, L, a.exact, cap, st, w.lp.tensor_cores);
            lp_build_symmetric(w.lp, L, cap, st);
            launched += 12;
        }
        launched += ppe_sp_enqueue_pack(w, a, cap, st, !(w.c16_learned && !a.batch.n));
    }
    return launched;
}

LpSystem ppe_lp_system(const PpeWork& w, const StageArgs& a) {
    LpSystem L;
    L.pos = w.pos_snap;
    L.n = w.n_snap;
    L.id = w.id_snap;
    L.rlen = w.rlen;
    L.diag64 = w.diag64;
    L.rowlist = w.rowlist;
    L.nrows = w.nrows;
    L.acols = w.cols;
    L.cell = a.cur.cell;
    L.cell_start = a.cell_start;
    L.g = a.g;
    L.P = a.P;
    L.sc = a.sc;
    if (a.batch.n) {
        L.sid_of_id = a.batch.sid_of_id;
        L.grids = a.batch.grid;
        L.phys = a.batch.phys;
    }
    return L;
}

int ppe_enable_learned(PpeWork& w, std::string* err) {
    if (w.lp.ready) return MPS_OK;
    return lp_setup(w.lp, w.cap, err);
}

int ppe_enqueue_solve(PpeWork& w, const StageArgs& a, const mps_options& opt, uint32_t cap, cudaStream_t st) {
    SolveArgs S;
    S.cols = w.cols;
    S.rlen = w.rlen;
    S.diag64 = w.diag64;
    S.diag32 = w.diag32;
    S.inv_diag = w.inv_diag;
    S.b64 = w.b64;
    S.x64 = w.x64;
    S.r = w.r;
    S.zp0 = w.zp[0];
    S.zp1 = w.zp[1];
    S.q = w.q;
    S.qp = w.qp;
    S.cap = cap;
    S.part = w.part;
    S.result = w.result;
    S.bar = w.bar;
    S.rowlist = w.rowlist;
    S.nrows = w.nrows;
    S.off = w.sell_off;
    S.scols = w.sell_cols;
    S.sw = w.sell_w;
    S.pos = a.cur.pos;
    S.rlap = a.P.rlap;
    S.rlap_thr = a.P.rlap_thr;
    S.sp_off = w.sp_off;
    S.sp_ent = w.sp_ent;
    S.sp_diag = w.sp_diag;
    S.rq0 = w.rq[0];
    S.rq1 = w.rq[1];
    S.sc = a.sc;
    S.tol = opt.cg_tol;
    S.max_iter = opt.cg_max_iter;
    S.inner_cap = opt.cg_check_every > 0 ? opt.cg_check_every : 500;
    S.eta_min = pow(10.0, -(double)(opt.cg_inner_digits > 0 ? opt.cg_inner_digits : 4));
    S.max_outer = 40;
    S.keep = w.l2_keep_entries;
    // shared-memory chunks (1 KB a warp each with stored weights): at most
    // PPE_SMEM_CHUNKS, 192 KB for the 32 warps of an SM
    S.smem_chunks = w.stored_weights ? (w.c16_smem_chunks < PPE_SMEM_CHUNKS ? w.c16_smem_chunks : PPE_SMEM_CHUNKS) : 0;
    if (S.smem_chunks < 0) S.smem_chunks = 0;
    if (a.batch.n) {
        BatchSolveArgs B;
        B.rowlist = w.rowlist;
        B.nrows = w.nrows;
        B.row_scene = w.row_scene;
        B.off = w.sell_off;
        B.scols = w.sell_cols;
        B.sw = w.sell_w;
        B.pos = a.cur.pos;
        B.phys = a.batch.phys;
        B.b64 = w.b64;
        B.diag64 = w.diag64;
        B.diag32 = w.diag32;
        B.inv_diag = w.inv_diag;
        B.x64 = w.x64;
        B.r = w.r;
        B.zp0 = w.zp[0];
        B.zp1 = w.zp[1];
        B.q = w.q;
        B.part = w.bpart;
        B.result = w.bresult;
        B.bar = w.bar;
        B.sc = a.sc;
        B.iters = w.scene_iters;
        B.outers = w.scene_outer;
        B.relres = w.scene_relres;
        B.ns = w.nscenes;
        B.tol = S.tol;
        B.max_iter = S.max_iter;
        B.inner_cap = S.inner_cap;
        B.max_outer = S.max_outer;
        B.eta_min = S.eta_min;
        B.keep = S.keep;
        B.sp_off = w.sp_off;
        B.sp_ent = w.sp_ent;
        B.sp_diag = w.sp_diag;
        B.rq0 = w.rq[0];
        B.rq1 = w.rq[1];
        void* bargs[] = {&B};
        const bool blearned = opt.precond == MPS_PRECOND_LEARNED && w.lp.ready && w.sp_ent;
        const void* bfn;
        if (blearned)
            bfn = w.stored_weights ? (a.exact ? (const void*)k_ppe_solve_batch<true, true, 1>
                                              : (const void*)k_ppe_solve_batch<false, true, 1>)
                                   : (a.exact ? (const void*)k_ppe_solve_batch<true, false, 1>
                                              : (const void*)k_ppe_solve_batch<false, false, 1>);
        else
            bfn = w.stored_weights ? (a.exact ? (const void*)k_ppe_solve_batch<true, true, 0>
                                              : (const void*)k_ppe_solve_batch<false, true, 0>)
                                   : (a.exact ? (const void*)k_ppe_solve_batch<true, false, 0>
                                              : (const void*)k_ppe_solve_batch<false, false, 0>);
        w.launch_err = launch_cooperative(bfn, w.blocks, w.threads, bargs, st);
        if (!w.write_pressure) return 1;
        k_ppe_finish<<<blocks_for(cap, 256), 256, 0, st>>>(w.x64, w.rlen, a.cur.press, a.sc);
        return 2;
    }
    const bool learned = opt.precond == MPS_PRECOND_LEARNED && w.lp.ready && w.sp_ent;
    if (w.c16 && (!learned || w.c16_learned)) return ppe_c16_enqueue_solve(w, a, opt, cap, st);
    if (w.pipelined && !learned) {
        PipeArgs Pa;
        Pa.rowlist = w.rowlist;
        Pa.nrows = w.nrows;
        Pa.off = w.sell_off;
        Pa.scols = w.sell_cols;
        Pa.sw = w.sell_w;
        Pa.pos = a.cur.pos;
        Pa.rlap = a.P.rlap;
        Pa.rlap_thr = a.P.rlap_thr;
        Pa.b64 = w.b64;
        Pa.diag64 = w.diag64;
        Pa.diag32 = w.diag32;
        Pa.inv_diag = w.inv_diag;
        Pa.x64 = w.x64;
        Pa.r = w.r;
        Pa.u = w.pu;
        Pa.w = w.pw;
        Pa.z = w.pz;
        Pa.q = w.pq;
        Pa.s = w.ps;
        Pa.p = w.pp;
        Pa.m0 = w.pm[0];
        Pa.m1 = w.pm[1];
        Pa.part = w.part;
        Pa.result = w.result;
        Pa.bar = w.bar;
        Pa.sc = a.sc;
        Pa.tol = S.tol;
        Pa.eta_min = S.eta_min;
        Pa.keep = S.keep;
        Pa.max_iter = S.max_iter;
        Pa.inner_cap = S.inner_cap;
        Pa.max_outer = S.max_outer;
        void* pargs[] = {&Pa};
        const void* pfn = w.stored_weights
                              ? (a.exact ? (const void*)k_ppe_solve_pipe<true, true> : (const void*)k_ppe_solve_pipe<false, true>)
                              : (a.exact ? (const void*)k_ppe_solve_pipe<true, false> : (const void*)k_ppe_solve_pipe<false, false>);
        w.launch_err = launch_cooperative(pfn, w.blocks, w.threads, pargs, st);
        if (!w.write_pressure) return 1;
        k_ppe_finish<<<blocks_for(cap, 256), 256, 0, st>>>(w.x64, w.rlen, a.cur.press, a.sc);
        return 2;
    }
    void* args[] = {&S};
    const void* fn;
    if (w.stored_weights)
        fn = a.exact ? (learned ? (const void*)k_ppe_solve<true, 1, true> : (const void*)k_ppe_solve<true, 0, true>)
                     : (learned ? (const void*)k_ppe_solve<false, 1, true> : (const void*)k_ppe_solve<false, 0, true>);
    else
        fn = a.exact ? (learned ? (const void*)k_ppe_solve<true, 1, false> : (const void*)k_ppe_solve<true, 0, false>)
                     : (learned ? (const void*)k_ppe_solve<false, 1, false> : (const void*)k_ppe_solve<false, 0, false>);
    const size_t smem = (size_t)(w.threads / 32) * (size_t)S.smem_chunks * 32 * (sizeof(uint4) + sizeof(float4));
    w.launch_err = launch_cooperative_smem(fn, w.blocks, w.threads, smem, args, st);
    if (!w.write_pressure) return 1;
    k_ppe_finish<<<blocks_for(cap, 256), 256, 0, st>>>(w.x64, w.rlen, a.cur.press, a.sc);
    return 2;
}

// ---------------------------------------------------------------- Crank-Nicolson viscosity
// MPS_CPU_IMPL::buildCG_CN<dir> (MPS_CAL_v4.0/MPS_CPU_IMPL.cpp:195-305) for
// velocity component c, on the PPE's data layout: a fluid row holds
//   A_ij = w_ij (fluid j), A_ii = -sum_j w_ij - 1/R,
//   b_i = -sum_j w_ij (u_j - u_i) - sum_{j boundary} w_ij u_j - u_i/R - dt g_c/R
// over every neighbour j != i within rlap (all types; w = rlap/r - 1), with
// 1/R = lambda n0 / (dim niu dt) and g the step's body force; other rows are
// Dirichlet (the reference's identity rows, x = u).  x starts at u.  One warp
// per particle scans the full 27 linked cells: components after the first
// see positions the earlier ones moved since the last cell rebuild, which
// the distance culling of the stage kernels does not allow for.
struct CnArgs {
    StageArgs a;
    int c;
    uint32_t* cols;
    float* wrm;
    uint32_t* rlen;
    double* diag64;
    float* diag32;
    float* inv_diag;
    double* b64;
    double* x64;
    unsigned* bar;
    double lambda_n0_over_dim_niu;  // lambda n0 / (dim niu): 1/R = this / dt
};

__device__ __forceinline__ float comp(const float4& v, int c) { return c == 0 ? v.x : (c == 1 ? v.y : v.z); }

template <bool EX>
__global__ void __launch_bounds__(256) k_cn_assemble(CnArgs A) {
    const StageArgs& a = A.a;
    const uint32_t n = a.sc->np;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (blockIdx.x == 0 && threadIdx.x == 0) A.bar[0] = 0u;  // the solver's barrier starts empty
    if (i >= n) return;
    const float4* __restrict__ pos = a.cur.pos;
    const float4* __restrict__ vel = a.cur.vel;
    const float4 pi = pos[i];
    const double ui = (double)comp(vel[i], A.c);
    if (ptype(pi) != T_FLUID) {
        if (lane == 0) {
            A.rlen[i] = PPE_DIRICHLET;
            A.diag64[i] = 1.0;
            A.diag32[i] = 1.0f;
            A.inv_diag[i] = 1.0f;
            A.b64[i] = ui;
            A.x64[i] = ui;
        }
        return;
    }
    const Local L = local_of<false>(a, i);
    const float re = a.P.rlap, thr = a.P.rlap_thr;
    uint32_t* cols = A.cols + (size_t)i * PPE_W;
    float* wrow = A.wrm + (size_t)i * PPE_W;
    uint32_t count = 0;
    double diag = 0.0, bi = 0.0;
    const uint32_t lt = (1u << lane) - 1u;
    const CellNear nr = cell_near(L.g, L.c, pi.x, pi.y, pi.z, re);
    walk_cells<!EX>(L.g, L.cs, L.c, nr, lane, [&](uint32_t j, bool in) {
        {
            bool app = false;
            float w = 0.f;
            if (in && j != i) {
                const float4 pj = __ldg(pos + j);
                const float dx = fsub<EX>(pj.x, pi.x), dy = fsub<EX>(pj.y, pi.y), dz = fsub<EX>(pj.z, pi.z);
                const float rr = dot3<EX>(dx, dy, dz, dx, dy, dz);
                if (rr < thr) w = weight_rr<EX>(re, rr);
                if (w > 0.f) {
                    const double uj = (double)comp(__ldg(vel + j), A.c);
                    bi -= (uj - ui) * (double)w;
                    if (ptype(pj) != T_FLUID) bi -= (double)w * uj;
                    else app = true;
                }
            }
            diag += (double)w;
            const uint32_t m = __ballot_sync(0xffffffffu, app);
            if (app) {
                const uint32_t k = count + __popc(m & lt);
                if (k < PPE_W) {
                    cols[k] = j;
                    wrow[k] = w;
                }
            }
            count += __popc(m);
        }
    });
    diag = warp_sum_d(diag);
    bi = warp_sum_d(bi);
    if (lane == 0) {
        if (count > PPE_W) {
            atomicOr(&a.sc->err, ERR_CAPACITY);
            count = PPE_W;
        }
        const double one_over_R = A.lambda_n0_over_dim_niu / (double)a.sc->dt;
        const double dg = -diag - one_over_R;
        A.rlen[i] = count;
        A.diag64[i] = dg;
        A.diag32[i] = (float)dg;
        A.inv_diag[i] = (float)(1.0 / dg);
        A.b64[i] = bi - (one_over_R * ui + A.lambda_n0_over_dim_niu * (double)a.sc->g_eff[A.c]);
        A.x64[i] = ui;
    }
}

// MPS_CPU_IMPL::updatePosVel<dir> (MPS_CAL_v4.0/MPS_CPU_IMPL.cpp:129-190):
// fluid u_c = x, x_c += dt u_c.
__global__ void k_cn_finish(const double* __restrict__ x64, const uint32_t* __restrict__ rlen, State s, int c,
                            const Scalars* sc) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= sc->np || rlen[i] == PPE_DIRICHLET) return;
    const float x = (float)x64[i];
    float4 u = s.vel[i], p = s.pos[i];
    const float np_ = __fadd_rn(comp(p, c), __fmul_rn(sc->dt, x));
    if (c == 0) { u.x = x; p.x = np_; }
    else if (c == 1) { u.y = x; p.y = np_; }
    else { u.z = x; p.z = np_; }
    s.vel[i] = u;
    s.pos[i] = p;
}

int ppe_enqueue_cn(PpeWork& w, const StageArgs& a, const mps_options& opt, int c, double n0, double lambda,
                   uint32_t cap, cudaStream_t st) {
    CnArgs A;
    A.a = a;
    A.c = c;
    A.cols = w.cols;
    A.wrm = w.wrm;
    A.rlen = w.rlen;
    A.diag64 = w.diag64;
    A.diag32 = w.diag32;
    A.inv_diag = w.inv_diag;
    A.b64 = w.b64;
    A.x64 = w.x64;
    A.bar = w.bar;
    A.lambda_n0_over_dim_niu = lambda * n0 / ((double)a.P.dim_f * (double)a.P.niu);
    const uint32_t warps_blocks = blocks_for(cap * 32u, 256);
    if (a.exact) k_cn_assemble<true><<<warps_blocks, 256, 0, st>>>(A);
    else k_cn_assemble<false><<<warps_blocks, 256, 0, st>>>(A);
    int launched = 1 + enqueue_rows_pack(w, a, cap, st);
    launched += ppe_enqueue_solve(w, a, opt, cap, st);
    k_cn_finish<<<blocks_for(cap, 256), 256, 0, st>>>(w.x64, w.rlen, a.cur, c, a.sc);
    return launched + 1;
}

int ppe_set_threads(PpeWork& w, int threads) {
    if (threads != 256 && threads != 512 && threads != 1024) return MPS_ERR_INVALID;
    const int per_sm = PPE_THREADS / threads;
    for (const void* f : solve_kernels()) {
        int o = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, f, threads, 0) != cudaSuccess || o < per_sm)
            return MPS_ERR_INVALID;
    }
    w.threads = threads;
    w.blocks = w.sms * per_sm;
    return MPS_OK;
}

int ppe_setup_batch(PpeWork& w, const PpeScene* scenes, uint32_t nscenes, cudaStream_t st, std::string* err) {
    if (nscenes == 0 || nscenes > PPE_MAX_SCENES) {
        *err = "a batch holds 1 to " + std::to_string(PPE_MAX_SCENES) + " scenes";
        return MPS_ERR_INVALID;
    }
    w.nscenes = nscenes;
    bool ok = true;
    auto al = [&](void** p, size_t bytes) {
        if (cudaMalloc(p, bytes + 64) != cudaSuccess) { ok = false; return; }
        cudaMemsetAsync(*p, 0, bytes + 64, st);
    };
    al((void**)&w.scenes, nscenes * sizeof(PpeScene));
    al((void**)&w.row_scene, (size_t)w.cap * sizeof(uint32_t));
    al((void**)&w.bpart, (size_t)w.sms * 4 * 3 * nscenes * sizeof(double));
    al((void**)&w.bresult, 3 * nscenes * sizeof(double));
    al((void**)&w.scene_iters, nscenes * sizeof(int));
    al((void**)&w.scene_outer, nscenes * sizeof(int));
    al((void**)&w.scene_relres, nscenes * sizeof(double));
    if (!ok) {
        *err = "cudaMalloc failed for the batch PPE tables";
        return MPS_ERR_CUDA;
    }
    if (cudaMemcpyAsync(w.scenes, scenes, nscenes * sizeof(PpeScene), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        *err = "upload of the batch PPE constants failed";
        return MPS_ERR_CUDA;
    }
    return MPS_OK;
}

void ppe_free(PpeWork& w) {
    void* ps[] = {w.cols, w.wrm, w.rlen, w.diag64, w.diag32, w.inv_diag, w.b64, w.x64,
                  w.r,    w.zp[0], w.zp[1], w.q,    w.qp,   w.part,     w.result, w.bar,
                  w.rowlist, w.tilecnt, w.nrows, w.sell_off, w.sell_cols, w.sell_w, w.pos_snap, w.n_snap,
                  w.id_snap, w.pu, w.pw, w.pz, w.pq, w.ps, w.pp, w.pm[0], w.pm[1], w.scenes, w.row_scene, w.bpart, w.bresult, w.scene_iters, w.scene_outer,
                  w.scene_relres, w.sp_off, w.sp_ent, w.sp_diag, w.rq[0], w.rq[1]};
    lp_free(w.lp);
    ppe_c16_free(w);
    for (void* p : ps)
        if (p) cudaFree(p);
    w = PpeWork();
}

}  // namespace mpsb
