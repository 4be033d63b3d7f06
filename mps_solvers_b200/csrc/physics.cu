// physics.cu -- particle stages of the MPS step on the sorted particles.
//
// One thread per particle walks the reference's 27 linked cells as 9 index
// ranges (link_row) in the reference's order.  Every stage writes its result
// to a separate array (tmp / n / press) and never to the positions or
// velocities it reads, which is the two-phase form of the reference's CPU
// stages; the second phase (u, x update) is applied by the following rebuild
// gather.  With EX = true each float operation is rounded once, in the
// reference's order, so the results equal the reference's CPU results.
#include "physics.cuh"
#include "cellsort.cuh"

namespace mpsb {

static inline uint32_t blocks_for(uint32_t n, uint32_t t) { return (n + t - 1) / t; }

// ---------------------------------------------------------------- gather
// dst[p] = src[perm[p]]; the pending update of a fluid particle is applied
// exactly as k_cell_keys applied it to find its cell; particles sorted past
// np_new (outside the grid) become type 3 with zero velocity and leave the
// active range (MPS_CAL_expl_v1.0/MPS_GPU.cpp:268-280, 329).
// A particle as the gathers move it: read from position `old` of src with
// the pending update of a fluid particle applied exactly as the keys kernel
// applied it to find its cell.  store_particle writes it to position p of
// dst; a key past the grid (left it) makes it type 3 at rest.  The merge
// gather loads before it knows p, so the loads overlap its searches.
struct Moved {
    float4 x, u;
    float press, n;
    uint32_t id;
};

__device__ __forceinline__ Moved load_particle(const State& src, uint32_t old, const float4* __restrict__ tmp,
                                               int apply, const Scalars* __restrict__ sc, const BatchDev& batch) {
    Moved v;
    v.x = src.pos[old];
    v.u = src.vel[old];
    v.press = src.press[old];
    v.n = src.n[old];
    v.id = src.id[old];
    if (apply != 0 && ptype(v.x) == T_FLUID) {
        const float dt = batch.n ? batch.dt[batch.sid_of_id[v.id]] : sc->dt;
        const float4 d = tmp[old];
        if (apply == 1) {
            v.u.x = d.x; v.u.y = d.y; v.u.z = d.z;
        } else {
            v.u.x = __fadd_rn(v.u.x, d.x); v.u.y = __fadd_rn(v.u.y, d.y); v.u.z = __fadd_rn(v.u.z, d.z);
        }
        v.x.x = __fadd_rn(v.x.x, __fmul_rn(dt, d.x));
        v.x.y = __fadd_rn(v.x.y, __fmul_rn(dt, d.y));
        v.x.z = __fadd_rn(v.x.z, __fmul_rn(dt, d.z));
    }
    return v;
}

// returns the particle's type
__device__ __forceinline__ uint32_t store_particle(const State& dst, Moved v, uint32_t p, uint32_t key,
                                                   uint32_t ncells, uint32_t* __restrict__ index_of_id) {
    if (key >= ncells) {  // left the grid
        v.x.w = __uint_as_float(T_EXCL);
        v.u = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    dst.pos[p] = v.x;
    dst.vel[p] = v.u;
    dst.press[p] = v.press;
    dst.n[p] = v.n;
    dst.id[p] = v.id;
    dst.cell[p] = key;
    index_of_id[v.id] = p;
    return ptype(v.x);
}

// The end of both gathers: this warp's particles (type ty, new position p)
// appended to the compact lists of the active fluid and non-dummy particles,
// then the last block to finish publishes the new active count.  The warps'
// runs land in the lists in the order the warps finish, which changes from
// run to run; every stage kernel treats its particles independently, except
// the fast viscosity, which pairs list entries 2w and 2w + 1.  Each warp's
// fluid run is therefore padded to an even length with a LIST_GAP entry, so
// that a pair never spans two runs and the pairs are the same in every run.
__device__ __forceinline__ void gather_tail(uint32_t ty, uint32_t p, uint32_t n, Scalars* __restrict__ sc,
                                            uint32_t* __restrict__ list_fluid, uint32_t* __restrict__ list_solid) {
    if (list_fluid) {
        const uint32_t lane = threadIdx.x & 31, lt = (1u << lane) - 1u;
        const bool f = ty == T_FLUID, s2 = ty == T_FLUID || ty == T_WALL;
        const uint32_t mf = __ballot_sync(0xffffffffu, f), ms = __ballot_sync(0xffffffffu, s2);
        uint32_t bf = 0, bs = 0;
        const uint32_t nf = __popc(mf);
        if (lane == 0) {
            if (mf) bf = atomicAdd(&sc->n_fluid, nf + (nf & 1u));
            if (ms) bs = atomicAdd(&sc->n_solid, __popc(ms));
        }
        bf = __shfl_sync(0xffffffffu, bf, 0);
        bs = __shfl_sync(0xffffffffu, bs, 0);
        if (f) list_fluid[bf + __popc(mf & lt)] = p;
        if (lane == 0 && (nf & 1u)) list_fluid[bf + nf] = LIST_GAP;
        if (s2) list_solid[bs + __popc(ms & lt)] = p;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const uint32_t done = atomicAdd(&sc->done_blocks, 1u);
        if (done == gridDim.x - 1) {
            __threadfence();
            const uint32_t nn = *(volatile uint32_t*)&sc->np_new;
            sc->nexcl += n - nn;
            sc->np = nn;
            sc->done_blocks = 0;
            __threadfence();
        }
    }
}

__global__ void __launch_bounds__(256) k_gather(State src, State dst, const uint32_t* __restrict__ perm,
                                                const uint32_t* __restrict__ keys_sorted,
                                                const float4* __restrict__ tmp, int apply,
                                                uint32_t* __restrict__ index_of_id, Scalars* __restrict__ sc,
                                                uint32_t* __restrict__ list_fluid, uint32_t* __restrict__ list_solid,
                                                BatchDev batch, uint32_t* __restrict__ cell_start, uint32_t ncells) {
    const uint32_t n = sc->np;
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    // the cell table (one thread per sorted position and one past the end)
    // and the count of particles inside the grid, whose keys sort first
    if (p <= n) {
        cell_start_fill(keys_sorted, n, ncells, p, cell_start);
        const long long prev = p > 0 ? (long long)keys_sorted[p - 1] : -1ll;
        const long long cur = p < n ? (long long)keys_sorted[p] : (long long)ncells;
        if (prev < (long long)ncells && cur >= (long long)ncells) sc->np_new = p;
    }
    uint32_t ty = T_EXCL;
    if (p < n)
        ty = store_particle(dst, load_particle(src, perm[p], tmp, apply, sc, batch), p, keys_sorted[p], ncells,
                            index_of_id);
    gather_tail(ty, p, n, sc, list_fluid, list_solid);
}

// The counts of entries below va in the ascending a[0..m) and below vb in
// the ascending b[0..m), searched in one loop so that the two searches'
// loads are in flight together
__device__ __forceinline__ void count_below2(const uint64_t* __restrict__ a, uint64_t va,
                                             const uint32_t* __restrict__ b, uint32_t vb, uint32_t m, uint32_t& ra,
                                             uint32_t& rb) {
    uint32_t alo = 0, ahi = m, blo = 0, bhi = m;
    while (alo < ahi || blo < bhi) {
        if (alo < ahi) {
            const uint32_t mid = (alo + ahi) >> 1;
            if (a[mid] < va) alo = mid + 1;
            else ahi = mid;
        }
        if (blo < bhi) {
            const uint32_t mid = (blo + bhi) >> 1;
            if (b[mid] < vb) blo = mid + 1;
            else bhi = mid;
        }
    }
    ra = alo;
    rb = blo;
}

// The merge rebuild's gather (cellsort.cuh): with B the changed particles'
// previous positions and A their (new key, previous position), both
// ascending, an unchanged particle at q goes to q - |B < q| + |A < (key, q)|
// and a changed one to its rank in A plus the unchanged particles before
// it, b - |B < b| with b = the first previous position past (key, q) in the
// old order; the new cell table is cs_old[c] - |B < cs_old[c]| +
// |A < (c, 0)|.  One thread per particle and per table entry.
__global__ void __launch_bounds__(256) k_merge_gather(State src, State dst, const uint32_t* __restrict__ newkey,
                                                      const uint64_t* __restrict__ a, const uint32_t* __restrict__ b,
                                                      const uint32_t* __restrict__ count,
                                                      const uint32_t* __restrict__ cs_old, uint32_t* __restrict__ cs_new,
                                                      uint32_t ncells, const float4* __restrict__ tmp, int apply,
                                                      uint32_t* __restrict__ index_of_id, Scalars* __restrict__ sc,
                                                      uint32_t* __restrict__ list_fluid,
                                                      uint32_t* __restrict__ list_solid, BatchDev batch) {
    const uint32_t n = sc->np;
    const uint32_t m = count[1];
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t <= ncells) {
        const uint32_t c0 = cs_old[t];
        uint32_t ra, rb;
        count_below2(a, (uint64_t)t << 32, b, c0, m, ra, rb);
        const uint32_t v = c0 - rb + ra;
        cs_new[t] = v;
        if (t == ncells) sc->np_new = v;
    }
    uint32_t ty = T_EXCL, p = 0;
    if (t < n) {
        const Moved v = load_particle(src, t, tmp, apply, sc, batch);
        const uint32_t k = newkey[t];
        const bool changed = k != src.cell[t];
        uint32_t bnd = t;  // the unchanged particle's own position
        if (changed) {
            const uint32_t lo = k < ncells ? cs_old[k] : n, hi = k < ncells ? cs_old[k + 1] : n;
            bnd = t < lo ? lo : (t > hi ? hi : t);
        }
        uint32_t ra, rb;
        count_below2(a, ((uint64_t)k << 32) | t, b, bnd, m, ra, rb);
        p = changed ? ra + bnd - rb : t - rb + ra;
        ty = store_particle(dst, v, p, k, ncells, index_of_id);
    }
    gather_tail(ty, p, n, sc, list_fluid, list_solid);
}

void launch_merge_gather(const State& src, const State& dst, const MergeScratch& m, const uint32_t* cs_old,
                         uint32_t* cs_new, uint32_t ncells, const float4* tmp, int apply, uint32_t* index_of_id,
                         Scalars* sc, uint32_t cap, cudaStream_t st, uint32_t* list_fluid, uint32_t* list_solid,
                         const BatchDev& batch) {
    const uint32_t threads = cap > ncells + 1 ? cap : ncells + 1;
    k_merge_gather<<<blocks_for(threads, 256), 256, 0, st>>>(src, dst, m.newkey, m.a, m.b, m.count, cs_old, cs_new,
                                                              ncells, tmp, apply, index_of_id, sc, list_fluid,
                                                              list_solid, batch);
}

void launch_gather(const State& src, const State& dst, const uint32_t* perm, const uint32_t* keys_sorted,
                   const float4* tmp, int apply, uint32_t* index_of_id, Scalars* sc, uint32_t cap, cudaStream_t st,
                   uint32_t* list_fluid, uint32_t* list_solid, const BatchDev& batch, uint32_t* cell_start,
                   uint32_t ncells) {
    k_gather<<<blocks_for(cap + 1, 256), 256, 0, st>>>(src, dst, perm, keys_sorted, tmp, apply, index_of_id, sc,
                                                        list_fluid, list_solid, batch, cell_start, ncells);
}

// ---------------------------------------------------------------- update_dt
// MPS_GPU::update_dt (MPS_CAL_expl_v1.0/MPS_GPU.cpp:761-777): dt = min over
// particles of CFL*dp/|u| (float CFL*dp divided by the double square root,
// rounded to float), capped at dt_max.  The minimum over particles is the
// value at the largest |u|^2, so a max-reduction of |u|^2 gives the same dt.
__global__ void __launch_bounds__(256) k_update_dt(const float4* __restrict__ vel, Phys P, Scalars* __restrict__ sc) {
    const uint32_t n = sc->np;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t m = 0;
    if (i < n) {
        const float4 u = vel[i];
        const float vv = dot3<true>(u.x, u.y, u.z, u.x, u.y, u.z);
        if (vv == vv) m = __float_as_uint(vv);
        else atomicOr(&sc->err, ERR_NAN);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m) atomicMax(&sc->vmax2_bits, m);
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const uint32_t done = atomicAdd(&sc->done_blocks, 1u);
        if (done == gridDim.x - 1) {
            __threadfence();
            const float vmax = __uint_as_float(atomicAdd(&sc->vmax2_bits, 0u));
            const float t = __double2float_rn((double)P.cfl_dp / sqrt((double)vmax));
            const float dt = t < P.dt_max ? t : P.dt_max;
            if (dt < P.dt_min) atomicOr(&sc->err, ERR_DT_TOO_SMALL);
            sc->dt = dt;
            body_force(P, sc->time, sc->g_eff);
            sc->vmax2_bits = 0;
            sc->done_blocks = 0;
            __threadfence();
        }
    }
}

// The same per scene of a batch: each scene's dt from its own largest |u|^2
// and constants, and its body force at its own time.
__global__ void __launch_bounds__(256) k_update_dt_batch(const float4* __restrict__ vel, const uint32_t* __restrict__ id,
                                                         BatchDev b, Scalars* __restrict__ sc) {
    const uint32_t n = sc->np;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const float4 u = vel[i];
        const float vv = dot3<true>(u.x, u.y, u.z, u.x, u.y, u.z);
        const uint32_t s = b.sid_of_id[id[i]];
        // lanes of the same scene (consecutive particles mostly share one)
        // combine before one atomic
        const uint32_t peers = __match_any_sync(__activemask(), s);
        uint32_t m = 0;
        if (vv == vv) m = __float_as_uint(vv);
        else atomicOr(&sc->err, ERR_NAN);
        uint32_t best = m;
        for (uint32_t rest = peers; rest;) {
            const int l = __ffs(rest) - 1;
            rest &= rest - 1u;
            best = max(best, __shfl_sync(peers, m, l));
        }
        if ((threadIdx.x & 31) == (uint32_t)(__ffs(peers) - 1) && best) atomicMax(b.vmax2_bits + s, best);
    }
    __syncthreads();
    __shared__ bool last;
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(&sc->done_blocks, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (uint32_t s = threadIdx.x; s < b.n; s += blockDim.x) {
        const Phys P = b.phys[s];
        const float vmax = __uint_as_float(atomicAdd(b.vmax2_bits + s, 0u));
        const float t = __double2float_rn((double)P.cfl_dp / sqrt((double)vmax));
        const float dt = t < P.dt_max ? t : P.dt_max;
        if (dt < P.dt_min) atomicOr(&sc->err, ERR_DT_TOO_SMALL);
        b.dt[s] = dt;
        float g[3];
        body_force(P, b.time[s], g);
        b.g_eff[s] = make_float4(g[0], g[1], g[2], 0.f);
        b.vmax2_bits[s] = 0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        sc->dt = b.dt[0];
        sc->done_blocks = 0;
        __threadfence();
    }
}

void launch_update_dt(const StageArgs& a, uint32_t cap, cudaStream_t st) {
    if (a.batch.n) k_update_dt_batch<<<blocks_for(cap, 256), 256, 0, st>>>(a.cur.vel, a.cur.id, a.batch, a.sc);
    else k_update_dt<<<blocks_for(cap, 256), 256, 0, st>>>(a.cur.vel, a.P, a.sc);
}

__global__ void k_step_end(Scalars* sc, BatchDev b) {
    sc->time = __fadd_rn(sc->time, sc->dt);
    sc->step += 1;
    for (uint32_t s = 0; s < b.n; s++) b.time[s] = __fadd_rn(b.time[s], b.dt[s]);
    if (b.n) sc->time = b.time[0];
}

void launch_step_end(Scalars* sc, const BatchDev& batch, cudaStream_t st) { k_step_end<<<1, 1, 0, st>>>(sc, batch); }

// ---------------------------------------------------------------- warp per particle
// One warp per particle; lane l takes candidate j = base + l of each row
// chunk.  ORD (explicit method, exact arithmetic): the warp adds the non-zero
// terms one by one in ascending lane (= ascending j) order, which is the
// reference's summation order, so the sums are bit-identical to its
// sequential loop.  Otherwise: lane-private partial sums and a fixed shuffle
// tree (deterministic, not the reference's order).
struct WarpTask {
    uint32_t i;      // particle
    bool ok;
};

__device__ __forceinline__ WarpTask warp_task(const StageArgs& a, const uint32_t* __restrict__ list,
                                              const uint32_t* __restrict__ list_n) {
    const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    WarpTask t;
    if (list) {
        const uint32_t n = *list_n;
        t.i = w < n ? list[w] : LIST_GAP;
        t.ok = t.i != LIST_GAP;
    } else {
        t.ok = w < a.sc->np;
        t.i = w;
    }
    return t;
}

// Ordered sums of one batch's terms (the reference adds a particle's
// neighbour terms one after another in candidate order).  The lanes with a
// term write it to the warp's shared buffer at its rank among them, and lane
// 0 adds the buffer in that order, one rounding per addition: the same
// additions as a loop over the hits, without a shuffle chain every lane runs.
// Only lane 0's sums are the result.  buf holds 32 entries per warp.
template <bool EX>
__device__ __forceinline__ void ordered_add1(float* buf, uint32_t lane, bool hit, float t, float& acc) {
    const uint32_t m = __ballot_sync(0xffffffffu, hit);
    if (m == 0u) return;
    if (hit) buf[__popc(m & ((1u << lane) - 1u))] = t;
    __syncwarp();
    if (lane == 0) {
        const int nh = __popc(m);
#pragma unroll 4
        for (int k = 0; k < nh; k++) acc = fadd<EX>(acc, buf[k]);
    }
    __syncwarp();
}

template <bool EX>
__device__ __forceinline__ void ordered_add3(float4* buf, uint32_t lane, bool hit, float tx, float ty, float tz,
                                             float& ax, float& ay, float& az) {
    const uint32_t m = __ballot_sync(0xffffffffu, hit);
    if (m == 0u) return;
    if (hit) buf[__popc(m & ((1u << lane) - 1u))] = make_float4(tx, ty, tz, 0.f);
    __syncwarp();
    if (lane == 0) {
        const int nh = __popc(m);
#pragma unroll 4
        for (int k = 0; k < nh; k++) {
            const float4 t = buf[k];
            ax = fadd<EX>(ax, t.x);
            ay = fadd<EX>(ay, t.y);
            az = fadd<EX>(az, t.z);
        }
    }
    __syncwarp();
}

// the warp's 32-entry buffer for ordered sums (blocks of up to 256 threads)
__device__ __forceinline__ float4* ordered_buf() {
    __shared__ float4 ord_buf[8][32];
    return ord_buf[(threadIdx.x >> 5) & 7u];
}

__device__ __forceinline__ float warp_tree_add(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <bool EX, bool ORD, bool BT>
__global__ void __launch_bounds__(256) k_visc_w(StageArgs a, const uint32_t* __restrict__ list,
                                                const uint32_t* __restrict__ list_n) {
    const WarpTask tk = warp_task(a, list, list_n);
    if (!tk.ok) return;
    const uint32_t i = tk.i, lane = threadIdx.x & 31;
    const float4* __restrict__ pos = a.cur.pos;
    const float4* __restrict__ vel = a.cur.vel;
    const float4 pi = pos[i];
    if (ptype(pi) != T_FLUID) return;
    const float4 ui = vel[i];
    const Local L = local_of<BT>(a, i);
    const Phys P = phys_of<BT>(a, L.s);
    const float re = P.rlap, thr = P.rlap_thr;
    float ax = 0.f, ay = 0.f, az = 0.f;
    float4* obuf = ordered_buf();
    const CellNear nr = cell_near(L.g, L.c, pi.x, pi.y, pi.z, re);
    walk_cells<!EX>(L.g, L.cs, L.c, nr, lane, [&](uint32_t j, bool in) {
        {
            float tx = 0.f, ty = 0.f, tz = 0.f;
            bool hit = false;
            if (in && j != i) {
                const float4 pj = __ldg(pos + j);
                const float dx = fsub<EX>(pj.x, pi.x), dy = fsub<EX>(pj.y, pi.y), dz = fsub<EX>(pj.z, pi.z);
                const float rr = dot3<EX>(dx, dy, dz, dx, dy, dz);
                if (rr < thr) {
                    const float w = weight_rr<EX>(re, rr);
                    if (w != 0.f) {
                        const float4 uj = __ldg(vel + j);
                        tx = fmul<EX>(w, fsub<EX>(uj.x, ui.x));
                        ty = fmul<EX>(w, fsub<EX>(uj.y, ui.y));
                        tz = fmul<EX>(w, fsub<EX>(uj.z, ui.z));
                        hit = true;
                    }
                }
            }
            if (ORD) ordered_add3<true>(obuf, lane, hit, tx, ty, tz, ax, ay, az);
            else { ax += tx; ay += ty; az += tz; }
        }
    });
    if (!ORD) { ax = warp_tree_add(ax); ay = warp_tree_add(ay); az = warp_tree_add(az); }
    if (lane != 0) return;
    const float dt = dt_of<BT>(a, L.s);
    float gx, gy, gz;
    if (BT) {
        const float4 ge = a.batch.g_eff[L.s];
        gx = ge.x; gy = ge.y; gz = ge.z;
    } else {
        gx = a.sc->g_eff[0]; gy = a.sc->g_eff[1]; gz = a.sc->g_eff[2];
    }
    const float lx = fmul<EX>(P.c_lap, ax), ly = fmul<EX>(P.c_lap, ay), lz = fmul<EX>(P.c_lap, az);
    float4 t;
    t.x = fadd<EX>(ui.x, fmul<EX>(dt, fadd<EX>(fmul<EX>(P.niu, lx), gx)));
    t.y = fadd<EX>(ui.y, fmul<EX>(dt, fadd<EX>(fmul<EX>(P.niu, ly), gy)));
    t.z = fadd<EX>(ui.z, fmul<EX>(dt, fadd<EX>(fmul<EX>(P.niu, lz), gz)));
    t.w = 0.f;
    a.tmp[i] = t;
}

// The unordered (fast) Laplacian for two fluid particles per warp: the
// warp walks the union of both particles' culled linked cells once and
// tests every candidate against both, so loads, index arithmetic and loop
// control are shared.  Used when the two list entries sit in the same cell
// (the common case: the fluid list is in sorted order within each warp of
// the gather); otherwise each particle walks its own cells.
template <bool BT>  // single scenes: 5 blocks an SM (48 registers) measured 5 % faster than 4
__global__ void __launch_bounds__(256, BT ? 3 : 5) k_visc_w2(StageArgs a, const uint32_t* __restrict__ list,
                                                 const uint32_t* __restrict__ list_n) {
    const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t nl = *list_n;
    if (2 * w >= nl) return;
    const uint32_t i1 = list[2 * w];  // never a gap: gaps sit at odd positions
    const uint32_t i2r = 2 * w + 1 < nl ? list[2 * w + 1] : LIST_GAP;
    const bool two = i2r != LIST_GAP;
    const uint32_t i2 = two ? i2r : i1;
    const float4* __restrict__ pos = a.cur.pos;
    const float4* __restrict__ vel = a.cur.vel;
    const float4 p1 = pos[i1], p2 = pos[i2];
    const float4 u1 = vel[i1], u2 = vel[i2];
    const Local L1 = local_of<BT>(a, i1);
    const Local L2 = local_of<BT>(a, i2);
    const Phys P = phys_of<BT>(a, L1.s);
    const float re = P.rlap, thr = P.rlap_thr;
    const bool shared = two && L1.c == L2.c && L1.s == L2.s;
    float a1x = 0.f, a1y = 0.f, a1z = 0.f, a2x = 0.f, a2y = 0.f, a2z = 0.f;
    const int rows = link_rows(L1.g);
    const CellNear n1 = cell_near(L1.g, L1.c, p1.x, p1.y, p1.z, re);
    const CellNear n2 = cell_near(L2.g, L2.c, p2.x, p2.y, p2.z, re);
    auto pair = [&](const float4& pi, const float4& ui, uint32_t i, uint32_t j, const float4& pj, const float4& uj,
                    float& ax, float& ay, float& az) {
        const float dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
        const float rr = dx * dx + dy * dy + dz * dz;
        if (j != i && rr < thr) {
            const float wgt = weight_rr<false>(re, rr);
            ax += wgt * (uj.x - ui.x);
            ay += wgt * (uj.y - ui.y);
            az += wgt * (uj.z - ui.z);
        }
    };
    if (shared) {
        auto both = [&](uint32_t j, bool in) {
            if (in) {
                const float4 pj = __ldg(pos + j), uj = __ldg(vel + j);
                pair(p1, u1, i1, j, pj, uj, a1x, a1y, a1z);
                pair(p2, u2, i2, j, pj, uj, a2x, a2y, a2z);
            }
        };
        // per row, the union of the two particles' culled ranges
        auto union_row = [&](int dz, int dy) {
            const RowRange r1 = link_row_near_at(L1.g, L1.cs, L1.c, dz, dy, n1);
            const RowRange r2 = link_row_near_at(L1.g, L1.cs, L1.c, dz, dy, n2);
            RowRange ru;
            ru.lo = r1.hi > r1.lo ? (r2.hi > r2.lo ? min(r1.lo, r2.lo) : r1.lo) : r2.lo;
            ru.hi = r1.hi > r1.lo ? (r2.hi > r2.lo ? max(r1.hi, r2.hi) : r1.hi) : r2.hi;
            return ru;
        };
        if (L1.g.reach > 1) {  // the refined grid: all rows as one list
            RowRange ru{0u, 0u};
            if ((int)lane < rows) {
                int dz, dy;
                row_offsets(L1.g, (int)lane, &dz, &dy);
                ru = union_row(dz, dy);
            }
            const FlatWalk fw = flat_walk_of(ru, lane);
            for (uint32_t f0 = 0; f0 < fw.total; f0 += 32) {
                const bool in = f0 + lane < fw.total;
                both(flat_at(fw, in ? f0 + lane : fw.total - 1), in);
            }
        } else {
            const int R = L1.g.reach, nz = L1.g.dim == 3 ? R : 0;
            for (int dz = -nz; dz <= nz; dz++)
                for (int dy = -R; dy <= R; dy++) {
                    const RowRange ru = union_row(dz, dy);
                    for (uint32_t base = ru.lo; base < ru.hi; base += 32) both(base + lane, base + lane < ru.hi);
                }
        }
    } else {
        for (int k = 0; k < (two ? 2 : 1); k++) {
            const Local& L = k ? L2 : L1;
            const CellNear& nr = k ? n2 : n1;
            const float4 pi = k ? p2 : p1, ui = k ? u2 : u1;
            const uint32_t i = k ? i2 : i1;
            float &ax = k ? a2x : a1x, &ay = k ? a2y : a1y, &az = k ? a2z : a1z;
            auto one = [&](uint32_t j, bool in) {
                if (in) pair(pi, ui, i, j, __ldg(pos + j), __ldg(vel + j), ax, ay, az);
            };
            if (L.g.reach > 1) walk_cells<true>(L.g, L.cs, L.c, nr, lane, one);
            else walk_cells<false>(L.g, L.cs, L.c, nr, lane, one);
        }
    }
    a1x = warp_tree_add(a1x); a1y = warp_tree_add(a1y); a1z = warp_tree_add(a1z);
    a2x = warp_tree_add(a2x); a2y = warp_tree_add(a2y); a2z = warp_tree_add(a2z);
    if (lane > 1 || (lane == 1 && !two)) return;
    const uint32_t i = lane ? i2 : i1;
    const float4 ui = lane ? u2 : u1;
    const Local& L = lane ? L2 : L1;
    const Phys Pi = phys_of<BT>(a, L.s);
    const float ax = lane ? a2x : a1x, ay = lane ? a2y : a1y, az = lane ? a2z : a1z;
    const float dt = dt_of<BT>(a, L.s);
    float gx, gy, gz;
    if (BT) {
        const float4 ge = a.batch.g_eff[L.s];
        gx = ge.x; gy = ge.y; gz = ge.z;
    } else {
        gx = a.sc->g_eff[0]; gy = a.sc->g_eff[1]; gz = a.sc->g_eff[2];
    }
    const float lx = Pi.c_lap * ax, ly = Pi.c_lap * ay, lz = Pi.c_lap * az;
    float4 t;
    t.x = ui.x + dt * (Pi.niu * lx + gx);
    t.y = ui.y + dt * (Pi.niu * ly + gy);
    t.z = ui.z + dt * (Pi.niu * lz + gz);
    t.w = 0.f;
    a.tmp[i] = t;
}

template <bool EX, bool ORD, bool BT>
__global__ void __launch_bounds__(256) k_collision_w(StageArgs a, const uint32_t* __restrict__ list,
                                                     const uint32_t* __restrict__ list_n) {
    const WarpTask tk = warp_task(a, list, list_n);
    if (!tk.ok) return;
    const uint32_t i = tk.i, lane = threadIdx.x & 31;
    const float4* __restrict__ pos = a.cur.pos;
    const float4* __restrict__ vel = a.cur.vel;
    const float4 pi = pos[i];
    if (ptype(pi) != T_FLUID) return;
    const float4 ui = vel[i];
    float cx = 0.f, cy = 0.f, cz = 0.f;
    float4* obuf = ordered_buf();
    const Local L = local_of<BT>(a, i);
    const Phys P = phys_of<BT>(a, L.s);
    const CellNear nr = cell_near(L.g, L.c, pi.x, pi.y, pi.z, P.col_dis);
    walk_cells<!EX>(L.g, L.cs, L.c, nr, lane, [&](uint32_t j, bool in) {
        {
            float tx = 0.f, ty = 0.f, tz = 0.f;
            bool hit = false;
            if (in && j != i) {
                const float4 pj = __ldg(pos + j);
                const float dx = fsub<EX>(pj.x, pi.x), dy = fsub<EX>(pj.y, pi.y), dz = fsub<EX>(pj.z, pi.z);
                const float rr = dot3<EX>(dx, dy, dz, dx, dy, dz);
                if (rr < P.col_thr) {
                    float ds, ood;
                    if (EX) { ds = __fsqrt_rn(rr); ood = __fdiv_rn(1.0f, ds); }
                    else { ood = rsqrtf(rr); ds = rr * ood; }
                    const float4 uj = __ldg(vel + j);
                    const float hx = fmul<EX>(0.5f, fsub<EX>(uj.x, ui.x));
                    const float hy = fmul<EX>(0.5f, fsub<EX>(uj.y, ui.y));
                    const float hz = fmul<EX>(0.5f, fsub<EX>(uj.z, ui.z));
                    const float vabs = fmul<EX>(dot3<EX>(hx, hy, hz, dx, dy, dz), ood);
                    if (ds <= P.col_dis && vabs <= 0.f) {
                        const float k = fmul<EX>(fmul<EX>(P.col_rate, vabs), ood);
                        tx = fmul<EX>(k, dx);
                        ty = fmul<EX>(k, dy);
                        tz = fmul<EX>(k, dz);
                        hit = true;
                    }
                }
            }
            if (ORD) ordered_add3<true>(obuf, lane, hit, tx, ty, tz, cx, cy, cz);
            else { cx += tx; cy += ty; cz += tz; }
        }
    });
    if (!ORD) { cx = warp_tree_add(cx); cy = warp_tree_add(cy); cz = warp_tree_add(cz); }
    if (lane == 0) a.tmp[i] = make_float4(cx, cy, cz, 0.f);
}

template <bool EX, bool ORD, bool BT>
__global__ void __launch_bounds__(256) k_pnd_w(StageArgs a, int eos, int all_types, const uint32_t* __restrict__ list,
                                               const uint32_t* __restrict__ list_n) {
    const WarpTask tk = warp_task(a, list, list_n);
    if (!tk.ok) return;
    const uint32_t i = tk.i, lane = threadIdx.x & 31;
    const float4* __restrict__ pos = a.cur.pos;
    const float4 pi = pos[i];
    if (!all_types && ptype(pi) == T_DUMMY) return;
    const Local L = local_of<BT>(a, i);
    const Phys P = phys_of<BT>(a, L.s);
    const float re = P.rzero, thr = P.rzero_thr;
    float acc = 0.f;
    float4* obuf = ordered_buf();
    const CellNear nr = cell_near(L.g, L.c, pi.x, pi.y, pi.z, re);
    walk_cells<!EX>(L.g, L.cs, L.c, nr, lane, [&](uint32_t j, bool in) {
        {
            float w = 0.f;
            if (in && j != i) {
                const float4 pj = __ldg(pos + j);
                const float dx = fsub<EX>(pj.x, pi.x), dy = fsub<EX>(pj.y, pi.y), dz = fsub<EX>(pj.z, pi.z);
                const float rr = dot3<EX>(dx, dy, dz, dx, dy, dz);
                if (rr < thr) w = weight_rr<EX>(re, rr);
            }
            if (ORD) ordered_add1<true>(reinterpret_cast<float*>(obuf), lane, w != 0.f, w, acc);
            else acc += w;
        }
    });
    if (!ORD) acc = warp_tree_add(acc);
    if (lane != 0) return;
    a.cur.n[i] = acc;
    if (eos) {
        const float t = fmul<EX>(fmul<EX>(P.one_over_alpha, fsub<EX>(acc, P.nzero)), P.one_over_nzero);
        a.cur.press[i] = t > 0.f ? t : 0.f;
    }
}

constexpr uint32_t DASH_SLOTS = 64;  // neighbours within r0 kept per particle (~32 on the lattice)

template <bool EX, bool ORD, bool BT>
__global__ void __launch_bounds__(256) k_dash_w(StageArgs a, const uint32_t* __restrict__ list,
                                                const uint32_t* __restrict__ list_n) {
    const WarpTask tk = warp_task(a, list, list_n);
    if (!tk.ok) return;
    const uint32_t i = tk.i, lane = threadIdx.x & 31;
    const float4* __restrict__ pos = a.cur.pos;
    const float* __restrict__ press = a.cur.press;
    const float4 pi = pos[i];
    if (ptype(pi) != T_FLUID) return;
    const Local L = local_of<BT>(a, i);
    const Phys P = phys_of<BT>(a, L.s);
    const float r02 = P.rzero2;
    const CellNear nr = cell_near(L.g, L.c, pi.x, pi.y, pi.z, P.rzero);
    // p_hat: a minimum, independent of order.  The same walk keeps every
    // candidate within r0 (any type, ascending index) in this warp's slots,
    // so the gradient below visits only those instead of walking the cells
    // again; more than DASH_SLOTS of them and it walks the cells again.
    __shared__ uint32_t slots[8][DASH_SLOTS];
    uint32_t* my = slots[(threadIdx.x >> 5) & 7u];
    const uint32_t lt = (1u << lane) - 1u;
    uint32_t nhit = 0;
    float hat = press[i];
    walk_cells<!EX>(L.g, L.cs, L.c, nr, lane, [&](uint32_t j, bool in) {
        {
            bool near = false;
            if (in) {
                const float4 pj = __ldg(pos + j);
                const float dx = fsub<EX>(pj.x, pi.x), dy = fsub<EX>(pj.y, pi.y), dz = fsub<EX>(pj.z, pi.z);
                const float rr = dot3<EX>(dx, dy, dz, dx, dy, dz);
                near = rr <= r02 || rr < P.rzero_thr;  // both passes' candidates
                if (rr <= r02 && ptype(pj) != T_DUMMY) {
                    const float pjv = __ldg(press + j);
                    if (pjv < hat) hat = pjv;
                }
            }
            const uint32_t m = __ballot_sync(0xffffffffu, near);
            if (near) {
                const uint32_t k = nhit + __popc(m & lt);
                if (k < DASH_SLOTS) my[k] = j;
            }
            nhit += __popc(m);
        }
    });
    __syncwarp();
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) hat = fminf(hat, __shfl_xor_sync(0xffffffffu, hat, o));
    const float re = P.rzero, thr = P.rzero_thr;
    const bool skip_dummy = a.semi != 0;
    float gx = 0.f, gy = 0.f, gz = 0.f;
    float4* obuf = ordered_buf();
    // the gradient's terms: candidates of the kept slots, in the same
    // ascending order as the cell walk, or the cell walk itself
    const bool slotted = nhit <= DASH_SLOTS;
    auto grad = [&](uint32_t j, bool in) {
        {
            float tx = 0.f, ty = 0.f, tz = 0.f;
            bool hit = false;
            if (in && j != i) {
                const float4 pj = __ldg(pos + j);
                if (!(skip_dummy && ptype(pj) == T_DUMMY)) {
                    const float dx = fsub<EX>(pj.x, pi.x), dy = fsub<EX>(pj.y, pi.y), dz = fsub<EX>(pj.z, pi.z);
                    const float rr = dot3<EX>(dx, dy, dz, dx, dy, dz);
                    if (rr < thr) {
                        const float w = weight_rr<EX>(re, rr);
                        if (w != 0.f) {
                            const float k = fmul<EX>(fdiv<EX>(fsub<EX>(__ldg(press + j), hat), rr), w);
                            tx = fmul<EX>(k, dx);
                            ty = fmul<EX>(k, dy);
                            tz = fmul<EX>(k, dz);
                            hit = true;
                        }
                    }
                }
            }
            if (ORD) ordered_add3<true>(obuf, lane, hit, tx, ty, tz, gx, gy, gz);
            else { gx += tx; gy += ty; gz += tz; }
        }
    };
    if (slotted) {
        for (uint32_t f0 = 0; f0 < nhit; f0 += 32) {
            const bool in = f0 + lane < nhit;
            grad(in ? my[f0 + lane] : 0xFFFFFFFFu, in);
        }
    } else {
        walk_cells<!EX>(L.g, L.cs, L.c, nr, lane, grad);
    }
    if (!ORD) { gx = warp_tree_add(gx); gy = warp_tree_add(gy); gz = warp_tree_add(gz); }
    if (lane != 0) return;
    const float cg = fmul<EX>(P.dim_f, P.one_over_nzero);
    const float kk = fmul<EX>(-dt_of<BT>(a, L.s), P.one_over_rho);
    a.tmp[i] = make_float4(fmul<EX>(kk, fmul<EX>(cg, gx)), fmul<EX>(kk, fmul<EX>(cg, gy)),
                           fmul<EX>(kk, fmul<EX>(cg, gz)), 0.f);
}

// ---------------------------------------------------------------- viscosity
// calVisc_expl + d3_LapVel (MPS_CAL_expl_v1.0/MPS_GPU_EXPL.cpp:344-386,
// MPS_GPU.cpp:683-717): for a fluid particle,
//   tmp = u + dt*(nu * c_lap * sum_j w(r; rlap) (u_j - u_i) + g).
void launch_visc(const StageArgs& a, uint32_t cap, cudaStream_t st) {
    const uint32_t nb = blocks_for((a.list_fluid ? a.cap_fluid : cap) * 32u, (uint32_t)a.threads);
    const uint32_t nb2 = blocks_for((a.cap_fluid + 1) / 2 * 32u, (uint32_t)a.threads);  // two particles a warp
    const bool ord = a.exact && !a.semi;
    if (a.batch.n) {
        if (a.exact && ord) k_visc_w<true, true, true><<<nb, a.threads, 0, st>>>(a, a.list_fluid, a.n_fluid);
        else if (a.exact) k_visc_w<true, false, true><<<nb, a.threads, 0, st>>>(a, a.list_fluid, a.n_fluid);
        else if (a.list_fluid) k_visc_w2<true><<<nb2, a.threads, 0, st>>>(a, a.list_fluid, a.n_fluid);
        else k_visc_w<false, false, true><<<nb, a.threads, 0, st>>>(a, a.list_fluid, a.n_fluid);
    } else {
        if (a.exact && ord) k_visc_w<true, true, false><<<nb, a.threads, 0, st>>>(a, a.list_fluid, a.n_fluid);
        else if (a.exact) k_visc_w<true, false, false><<<nb, a.threads, 0, st>>>(a, a.list_fluid, a.n_fluid);
        else if (a.list_fluid) k_visc_w2<false><<<nb2, a.threads, 0, st>>>(a, a.list_fluid, a.n_fluid);
        else k_visc_w<false, false, false><<<nb, a.threads, 0, st>>>(a, a.list_fluid, a.n_fluid);
    }
}

// ---------------------------------------------------------------- collision
// MPS_GPU::collision (MPS_CAL_expl_v1.0/MPS_GPU.cpp:892-986): for a fluid
// particle, over neighbours of any type with ds <= col_dis that approach
// (vabs = (0.5 du).dr / ds <= 0): crt += col_rate * vabs / ds * dr.
void launch_collision(const StageArgs& a, uint32_t cap, cudaStream_t st) {
    const uint32_t nb = blocks_for((a.list_fluid ? a.cap_fluid : cap) * 32u, (uint32_t)a.threads);
    const bool ord = a.exact && !a.semi;
    if (a.batch.n) {
        if (a.exact && ord) k_collision_w<true, true, true><<<nb, a.threads, 0, st>>>(a, a.list_fluid, a.n_fluid);
        else if (a.exact) k_collision_w<true, false, true><<<nb, a.threads, 0, st>>>(a, a.list_fluid, a.n_fluid);
        else k_collision_w<false, false, true><<<nb, a.threads, 0, st>>>(a, a.list_fluid, a.n_fluid);
    } else {
        if (a.exact && ord) k_collision_w<true, true, false><<<nb, a.threads, 0, st>>>(a, a.list_fluid, a.n_fluid);
        else if (a.exact) k_collision_w<true, false, false><<<nb, a.threads, 0, st>>>(a, a.list_fluid, a.n_fluid);
        else k_collision_w<false, false, false><<<nb, a.threads, 0, st>>>(a, a.list_fluid, a.n_fluid);
    }
}

// ---------------------------------------------------------------- PND (+EOS)
// cal_n (MPS_CAL_expl_v1.0/MPS_GPU.cpp:830-887): n_i = sum_{j != i} w(r; r0)
// for type != 2 (all types during initialisation, MPS.cpp:433-497), and the
// equation of state of calPres_expl (MPS_GPU_EXPL.cpp:391-415):
//   p = max(0, rho c^2 (n - n0) / n0).
void launch_pnd(const StageArgs& a, int eos, int all_types, uint32_t cap, cudaStream_t st) {
    const bool use_list = a.list_solid && !all_types;
    const uint32_t* list = use_list ? a.list_solid : nullptr;
    const uint32_t nb = blocks_for((use_list ? a.cap_solid : cap) * 32u, (uint32_t)a.threads);
    const bool ord = a.exact && !a.semi;
    if (a.batch.n) {
        if (a.exact && ord) k_pnd_w<true, true, true><<<nb, a.threads, 0, st>>>(a, eos, all_types, list, a.n_solid);
        else if (a.exact) k_pnd_w<true, false, true><<<nb, a.threads, 0, st>>>(a, eos, all_types, list, a.n_solid);
        else k_pnd_w<false, false, true><<<nb, a.threads, 0, st>>>(a, eos, all_types, list, a.n_solid);
    } else {
        if (a.exact && ord) k_pnd_w<true, true, false><<<nb, a.threads, 0, st>>>(a, eos, all_types, list, a.n_solid);
        else if (a.exact) k_pnd_w<true, false, false><<<nb, a.threads, 0, st>>>(a, eos, all_types, list, a.n_solid);
        else k_pnd_w<false, false, false><<<nb, a.threads, 0, st>>>(a, eos, all_types, list, a.n_solid);
    }
}

// calPres_expl second loop (MPS_CAL_expl_v1.0/MPS_GPU_EXPL.cpp:417-426): a
// type-2 particle takes the pressure of its wall particle i_normal.
__global__ void __launch_bounds__(256) k_dummy_press(State s, const uint32_t* __restrict__ normal_id_of,
                                                     const uint32_t* __restrict__ index_of_id,
                                                     const Scalars* __restrict__ sc) {
    const uint32_t n = sc->np;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (ptype(s.pos[i]) != T_DUMMY) return;
    const uint32_t j = index_of_id[normal_id_of[s.id[i]]];
    s.press[i] = s.press[j];
}

void launch_dummy_press(const StageArgs& a, const uint32_t* normal_id_of, const uint32_t* index_of_id, uint32_t cap,
                        cudaStream_t st) {
    k_dummy_press<<<blocks_for(cap, 256), 256, 0, st>>>(a.cur, normal_id_of, index_of_id, a.sc);
}

// ---------------------------------------------------------------- gradient
// calDash + d3_GradPres (MPS_CAL_expl_v1.0/MPS_GPU.cpp:571-638, 782-825): for
// a fluid particle, p_hat = min p over type != 2 neighbours with r^2 <= r0^2
// (itself included), grad = d/n0 * sum_{j != i} (p_j - p_hat)/r^2 w(r; r0) dr
// over every type (semi-implicit: type 2 excluded, MPS_CAL_v4.0/MPS_CPU.cpp:384-445),
// tmp = -dt/rho * grad.
void launch_dash(const StageArgs& a, uint32_t cap, cudaStream_t st) {
    const uint32_t nb = blocks_for((a.list_fluid ? a.cap_fluid : cap) * 32u, (uint32_t)a.threads);
    const bool ord = a.exact && !a.semi;
    if (a.batch.n) {
        if (a.exact && ord) k_dash_w<true, true, true><<<nb, a.threads, 0, st>>>(a, a.list_fluid, a.n_fluid);
        else if (a.exact) k_dash_w<true, false, true><<<nb, a.threads, 0, st>>>(a, a.list_fluid, a.n_fluid);
        else k_dash_w<false, false, true><<<nb, a.threads, 0, st>>>(a, a.list_fluid, a.n_fluid);
    } else {
        if (a.exact && ord) k_dash_w<true, true, false><<<nb, a.threads, 0, st>>>(a, a.list_fluid, a.n_fluid);
        else if (a.exact) k_dash_w<true, false, false><<<nb, a.threads, 0, st>>>(a, a.list_fluid, a.n_fluid);
        else k_dash_w<false, false, false><<<nb, a.threads, 0, st>>>(a, a.list_fluid, a.n_fluid);
    }
}

// ---------------------------------------------------------------- staging
__global__ void __launch_bounds__(256) k_fill_excluded(Staging o, uint32_t np0) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= np0) return;
    o.id[k] = k;
    o.type[k] = T_EXCL;
    o.press[k] = 0.f;
    o.n[k] = 0.f;
    for (int c = 0; c < 3; c++) {
        o.pos3[3 * k + c] = 0.f;
        o.vel3[3 * k + c] = 0.f;
    }
}

__global__ void __launch_bounds__(256) k_unpack(State s, Staging o, int by_id, uint32_t np0,
                                                const Scalars* __restrict__ sc) {
    const uint32_t n = sc->np;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 x = s.pos[i], u = s.vel[i];
    const uint32_t id = s.id[i];
    uint32_t k = i;
    if (by_id) {
        if (id >= np0) return;
        k = id;
    }
    o.id[k] = id;
    o.type[k] = ptype(x);
    o.pos3[3 * k] = x.x; o.pos3[3 * k + 1] = x.y; o.pos3[3 * k + 2] = x.z;
    o.vel3[3 * k] = u.x; o.vel3[3 * k + 1] = u.y; o.vel3[3 * k + 2] = u.z;
    o.press[k] = s.press[i];
    o.n[k] = s.n[i];
}

__global__ void __launch_bounds__(256) k_pack(State s, Staging in, int mask, const Scalars* __restrict__ sc) {
    const uint32_t n = sc->np;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (mask & 1) {
        float4 x = s.pos[i];
        x.x = in.pos3[3 * i]; x.y = in.pos3[3 * i + 1]; x.z = in.pos3[3 * i + 2];
        s.pos[i] = x;
    }
    if (mask & 2) {
        float4 u = s.vel[i];
        u.x = in.vel3[3 * i]; u.y = in.vel3[3 * i + 1]; u.z = in.vel3[3 * i + 2];
        s.vel[i] = u;
    }
    if (mask & 4) s.press[i] = in.press[i];
    if (mask & 8) s.n[i] = in.n[i];
}

void launch_unpack(const State& s, const Staging& out, int by_id, uint32_t np0, const Scalars* sc, uint32_t cap,
                   cudaStream_t st) {
    if (by_id) k_fill_excluded<<<blocks_for(np0, 256), 256, 0, st>>>(out, np0);
    k_unpack<<<blocks_for(cap, 256), 256, 0, st>>>(s, out, by_id, np0, sc);
}

void launch_pack(const State& s, const Staging& in, int mask, const Scalars* sc, uint32_t cap, cudaStream_t st) {
    k_pack<<<blocks_for(cap, 256), 256, 0, st>>>(s, in, mask, sc);
}

// ---------------------------------------------------------------- init
// n0 = first maximum of n in index order (MPS_CAL_expl_v1.0/MPS.cpp:487-496):
// max over (n bits << 32 | ~index), n >= 0 so its bits order like its value.
__global__ void __launch_bounds__(256) k_nzero(const float* __restrict__ n, const Scalars* __restrict__ sc,
                                               unsigned long long* best) {
    const uint32_t np = sc->np;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long v = 0ull;
    if (i < np) v = ((unsigned long long)__float_as_uint(n[i]) << 32) | (unsigned long long)(0xffffffffu - i);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long t = __shfl_xor_sync(0xffffffffu, v, o);
        v = t > v ? t : v;
    }
    if ((threadIdx.x & 31) == 0 && v) atomicMax(best, v);
}

void launch_nzero(const float* n, Scalars* sc, unsigned long long* best, uint32_t cap, cudaStream_t st) {
    k_nzero<<<blocks_for(cap, 256), 256, 0, st>>>(n, sc, best);
}

__global__ void __launch_bounds__(256) k_nzero_range(const float* __restrict__ n, uint32_t lo, uint32_t hi,
                                                     unsigned long long* best) {
    const uint32_t i = lo + blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long v = 0ull;
    if (i < hi) v = ((unsigned long long)__float_as_uint(n[i]) << 32) | (unsigned long long)(0xffffffffu - i);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long t = __shfl_xor_sync(0xffffffffu, v, o);
        v = t > v ? t : v;
    }
    if ((threadIdx.x & 31) == 0 && v) atomicMax(best, v);
}

void launch_nzero_range(const float* n, uint32_t lo, uint32_t hi, unsigned long long* best, cudaStream_t st) {
    if (hi > lo) k_nzero_range<<<blocks_for(hi - lo, 256), 256, 0, st>>>(n, lo, hi, best);
}

// lambda (MPS_CAL_expl_v1.0/MPS.cpp:500-515): sum over i != t of
// r^2 w(r; r0), r = |x_i - x_t|, in index order; only the linked cells of t
// can hold non-zero terms and they are visited in ascending index order.
__global__ void k_lambda(StageArgs a, const unsigned long long* best, float* out) {
    const uint32_t t = 0xffffffffu - (uint32_t)(*best & 0xffffffffull);
    const float4 pt = a.cur.pos[t];
    const Local L = local_of(a, t);
    const Phys P = phys_of(a, L.s);
    float lam = 0.f;
    const int rows = link_rows(L.g);
    const CellNear nr = cell_near(L.g, L.c, pt.x, pt.y, pt.z, P.rzero);
    for (int row = 0; row < rows; row++) {
        const RowRange rg = link_row_near(L.g, L.cs, L.c, row, nr);
        for (uint32_t j = rg.lo; j < rg.hi; j++) {
            if (j == t) continue;
            const float4 pj = a.cur.pos[j];
            const float dx = __fsub_rn(pj.x, pt.x), dy = __fsub_rn(pj.y, pt.y), dz = __fsub_rn(pj.z, pt.z);
            const float rr = dot3<true>(dx, dy, dz, dx, dy, dz);
            const float r = __fsqrt_rn(rr);
            const float w = r < P.rzero ? __fsub_rn(__fdiv_rn(P.rzero, r), 1.0f) : 0.f;
            lam = __fadd_rn(lam, __fmul_rn(__fmul_rn(r, r), w));
        }
    }
    *out = lam;
}

void launch_lambda(const StageArgs& a, const unsigned long long* best, float* lambda_out, cudaStream_t st) {
    k_lambda<<<1, 1, 0, st>>>(a, best, lambda_out);
}

// i_normal (MPS_CAL_expl_v1.0/MPS.cpp:531-555): for a type-2 particle the
// first type-1 particle in index order that improves r^2 below 2 r0^2.
// `reach` cells along x and `reach_yz` along y and z cover sqrt(2) r0; rows
// are visited in ascending cell order, so candidates come in ascending index
// order.
__global__ void __launch_bounds__(256) k_normals(StageArgs a, int reach, int reach_yz,
                                                 uint32_t* __restrict__ normal_id_of) {
    const uint32_t n = a.sc->np;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 pi = a.cur.pos[i];
    const uint32_t idi = a.cur.id[i];
    if (ptype(pi) != T_DUMMY) {
        normal_id_of[idi] = idi;
        return;
    }
    const Local L = local_of(a, i);
    const Phys P = phys_of(a, L.s);
    float dis = __fmul_rn(__fmul_rn(2.0f, P.rzero), P.rzero);
    uint32_t best = 0xffffffffu;
    const uint32_t c = L.c;
    const Grid& g = L.g;
    const int nz = g.dim == 3 ? reach_yz : 0;
    for (int dz = -nz; dz <= nz; dz++) {
        for (int dy = -reach_yz; dy <= reach_yz; dy++) {
            const uint32_t c0 = c + (uint32_t)dz * g.sheet + (uint32_t)dy * g.cdx;
            uint32_t first = 0xffffffffu, last = 0;
            for (int dx = -reach; dx <= reach; dx++) {
                const uint32_t cc = c0 + (uint32_t)dx;
                if (cc < g.ncells) {
                    if (first == 0xffffffffu) first = cc;
                    last = cc;
                }
            }
            if (first == 0xffffffffu) continue;
            const uint32_t lo = L.cs[first], hi = L.cs[last + 1];
            for (uint32_t j = lo; j < hi; j++) {
                const float4 pj = a.cur.pos[j];
                if (ptype(pj) != T_WALL) continue;
                const float dx = __fsub_rn(pj.x, pi.x), dy2 = __fsub_rn(pj.y, pi.y), dz2 = __fsub_rn(pj.z, pi.z);
                const float rr = dot3<true>(dx, dy2, dz2, dx, dy2, dz2);
                if (rr < dis) {
                    dis = rr;
                    best = j;
                }
            }
        }
    }
    normal_id_of[idi] = best == 0xffffffffu ? idi : a.cur.id[best];
}

void launch_normals(const StageArgs& a, int reach, int reach_yz, uint32_t* normal_id_of, uint32_t cap,
                    cudaStream_t st) {
    k_normals<<<blocks_for(cap, 256), 256, 0, st>>>(a, reach, reach_yz, normal_id_of);
}

// ---------------------------------------------------------------- boundary motion
// The reference's hook MOTION::doMotion(pos, vel, np) (MPS_CAL_/MOTION.cpp:11-16,
// an empty loop there) is called by MPS_GPU::motion (MPS_CAL_/MPS_GPU.cpp:
// 1670-1673) as the first, commented-out statement of a step, followed by
// divideCell (MPS_CAL_/MPS_GPU_EXPL.cpp:93-95).  This is one concrete motion
// law for it; the arithmetic is spelled out (no contraction) so it matches
// the oracle's double expressions.
__global__ void k_motion_select(State s, const Scalars* sc, float3 lo, float3 hi, uint32_t m,
                                uint32_t* __restrict__ motion_of, float4* __restrict__ x0, uint32_t* count) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= sc->np) return;
    const float4 p = s.pos[i];
    const uint32_t t = ptype(p);
    if (t != T_WALL && t != T_DUMMY) return;
    if (p.x < lo.x || p.x > hi.x || p.y < lo.y || p.y > hi.y || p.z < lo.z || p.z > hi.z) return;
    const uint32_t id = s.id[i];
    if (motion_of[id] != NO_MOTION) return;
    motion_of[id] = m;
    x0[id] = p;
    atomicAdd(count, 1u);
}

__global__ void k_motion(State s, const Scalars* sc, const uint32_t* __restrict__ motion_of,
                         const float4* __restrict__ x0, MotionSet M) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= sc->np) return;
    const uint32_t m = motion_of[s.id[i]];
    if (m == NO_MOTION) return;
    const float4 a = x0[s.id[i]];
    const double tau = __dsub_rn((double)sc->time, M.t0[m]);
    const double arg = __dadd_rn(__dmul_rn(M.omega[m], tau), M.phase[m]);
    const double sn = __dsub_rn(sin(arg), sin(M.phase[m]));
    const double cs = __dmul_rn(M.omega[m], cos(arg));
    const double xa[3] = {(double)a.x, (double)a.y, (double)a.z};
    float xn[3], un[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        xn[c] = (float)__dadd_rn(__dadd_rn(xa[c], __dmul_rn(M.vel[m][c], tau)), __dmul_rn(M.amp[m][c], sn));
        un[c] = (float)__dadd_rn(M.vel[m][c], __dmul_rn(M.amp[m][c], cs));
    }
    const float4 p = s.pos[i];
    s.pos[i] = make_float4(xn[0], xn[1], xn[2], p.w);
    s.vel[i] = make_float4(un[0], un[1], un[2], s.vel[i].w);
}

__global__ void k_motion_stop(State s, const Scalars* sc, const uint32_t* __restrict__ motion_of) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= sc->np || motion_of[s.id[i]] == NO_MOTION) return;
    s.vel[i] = make_float4(0.f, 0.f, 0.f, s.vel[i].w);
}

void launch_motion_stop(const State& s, const Scalars* sc, const uint32_t* motion_of, uint32_t cap, cudaStream_t st) {
    k_motion_stop<<<blocks_for(cap, 256), 256, 0, st>>>(s, sc, motion_of);
}

void launch_motion_select(const State& s, const Scalars* sc, const float lo[3], const float hi[3], uint32_t m,
                          uint32_t* motion_of, float4* x0, uint32_t* count, uint32_t cap, cudaStream_t st) {
    k_motion_select<<<blocks_for(cap, 256), 256, 0, st>>>(s, sc, make_float3(lo[0], lo[1], lo[2]),
                                                         make_float3(hi[0], hi[1], hi[2]), m, motion_of, x0, count);
}

void launch_motion(const State& s, const Scalars* sc, const uint32_t* motion_of, const float4* x0,
                   const MotionSet& M, uint32_t cap, cudaStream_t st) {
    k_motion<<<blocks_for(cap, 256), 256, 0, st>>>(s, sc, motion_of, x0, M);
}

}  // namespace mpsb
