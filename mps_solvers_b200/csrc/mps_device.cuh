// mps_device.cuh -- device-side types and helpers shared by the kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace mpsb {

// Cell grid of the reference's cell list (MPS_CAL_expl_v1.0/MPS.cpp:567-642).
// The fast-arithmetic 3-D path halves the cells along y and z (cell_yz =
// cell_size / 2, twice the cells along y and z, reach 2): a walk then visits
// up to 25 rows of 3 half-height cells instead of 9 rows of 3 cells, and on
// a dam-break state the culled walk holds about 35 % fewer candidates for the
// rlap stencil and half as many for r0.  The reference's grid has cell_yz =
// cell_size and reach 1.
struct Grid {
    float left, back, bottom, cell_size;
    uint32_t cdx, cdy, cdz, sheet, ncells;
    int dim;
    uint32_t base;  // first global cell id of this grid (scenes of a batch; 0 otherwise)
    float cell_yz;  // cell edge along y and z (cell_size along x)
    int reach;      // cell rows walked on each side along y and z to cover cell_size
};

// Per-scene constants, fixed after initialisation.
struct Phys {
    float rzero, rlap, col_dis, col_rate, niu, rho, one_over_rho;
    float nzero, one_over_nzero, one_over_alpha, c_lap, dim_f;
    float dt_max, dt_min, cfl_dp, beta;
    float g[3];
    // prefilter thresholds on r^2: any r^2 at or above them is certainly
    // outside the corresponding test (see host set-up)
    float rzero_thr, rlap_thr, col_thr, rzero2;
    // PPE (semi-implicit)
    float lambda, alpha, one_over_dt_fixed;
    // tank acceleration a(t) = body_amp sin(body_omega t) along x; the body
    // force of the viscosity stage is g - a(t)
    double body_amp, body_omega;
};

// Device-resident per-step scalars (one instance per handle).
struct Scalars {
    float dt;              // dt of the current step
    float time;            // simulated time
    uint32_t np;           // active particles (the reference's i_np)
    uint32_t np_new;       // active particles after the running rebuild
    uint32_t nexcl;        // total dropped particles
    uint32_t vmax2_bits;   // max |u|^2 of the running update_dt (float bits)
    uint32_t err;          // sticky error bits (ERR_*)
    uint32_t done_blocks;  // last-block counter for reductions
    int step;
    int cg_iters;
    double cg_relres;
    uint32_t n_fluid;      // entries of the fluid list built by the last rebuild
    uint32_t n_solid;      // entries of the fluid + wall list
    int cg_outer;          // FP64 true-residual passes of the last PPE solve
    int pad_i;
    float g_eff[3];        // body force of the current step: g - a(time)
    float pad_f;
    // longest spin of one grid-wide wait before it gives up with
    // ERR_DEVICE_TIMEOUT (ns; 0: the default, 1 s); set by the host
    unsigned long long wait_ns;
};

constexpr unsigned long long DEFAULT_WAIT_NS = 1000000000ull;

// the wait budget of the grid-wide barriers, read once per wait
__device__ __forceinline__ unsigned long long wait_budget_ns(const Scalars* sc) {
    const unsigned long long w = __ldcg(&sc->wait_ns);
    return w ? w : DEFAULT_WAIT_NS;
}

// The scenes of a batch: one particle set and one cell space made of each
// scene's own particles and cell grid, with per-scene constants and step
// scalars.  n == 0 (the default) is a single scene, and no array is read.
struct BatchDev {
    uint32_t n = 0;
    const uint32_t* sid_of_id = nullptr;  // scene of each particle id
    const Grid* grid = nullptr;           // per scene; base = its first global cell
    const Phys* phys = nullptr;           // per scene
    float* dt = nullptr;                  // per scene: dt of the current step
    float* time = nullptr;                // per scene: simulated time
    float4* g_eff = nullptr;              // per scene: g - a(time) of the current step
    uint32_t* vmax2_bits = nullptr;       // per scene: max |u|^2 of the running update_dt
    uint32_t ncells = 0;                  // cells of all scenes (the sentinel key)
};

// g - a(t) with a(t) = body_amp sin(body_omega t) along x, each component
// rounded once to float; exactly g when there is no tank acceleration.
__device__ __forceinline__ void body_force(const Phys& P, float t, float out[3]) {
    out[0] = P.g[0];
    out[1] = P.g[1];
    out[2] = P.g[2];
    if (P.body_amp != 0.0) out[0] = (float)((double)P.g[0] - P.body_amp * sin(P.body_omega * (double)t));
}

enum : uint32_t {
    ERR_DT_TOO_SMALL = 1u,
    ERR_NAN = 2u,
    ERR_PARTICLE_OUT = 4u,
    ERR_CG_NOT_CONVERGED = 8u,
    ERR_DEVICE_TIMEOUT = 16u,
    ERR_CAPACITY = 32u,
};

// particle types (pos.w carries the type as its bit pattern)
enum : uint32_t { T_FLUID = 0, T_WALL = 1, T_DUMMY = 2, T_EXCL = 3 };

__device__ __forceinline__ uint32_t ptype(const float4& p) { return __float_as_uint(p.w); }

// ---- arithmetic: EX = true evaluates in IEEE float, one rounding per
// operation, no contraction (the reference's SSE evaluation); EX = false lets
// the compiler fuse and uses approximate reciprocals.
template <bool EX> __device__ __forceinline__ float fmul(float a, float b) { return EX ? __fmul_rn(a, b) : a * b; }
template <bool EX> __device__ __forceinline__ float fadd(float a, float b) { return EX ? __fadd_rn(a, b) : a + b; }
template <bool EX> __device__ __forceinline__ float fsub(float a, float b) { return EX ? __fsub_rn(a, b) : a - b; }
template <bool EX> __device__ __forceinline__ float fdiv(float a, float b) { return EX ? __fdiv_rn(a, b) : __fdividef(a, b); }

// r.r summed x, y, z in that order (real3 operator*, typedef.h:103-106)
template <bool EX> __device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz) {
    return fadd<EX>(fadd<EX>(fmul<EX>(ax, bx), fmul<EX>(ay, by)), fmul<EX>(az, bz));
}

// d_weight(re, sqrt(rr)) = re/r - 1 for r < re (MPS_CAL_expl_v1.0/MPS.cpp:412-417),
// given rr below the prefilter threshold.  Returns 0 outside.
template <bool EX> __device__ __forceinline__ float weight_rr(float re, float rr) {
    if (EX) {
        float r = __fsqrt_rn(rr);
        return r < re ? __fsub_rn(__fdiv_rn(re, r), 1.0f) : 0.0f;
    } else {
        return rr < re * re ? fmaf(re, rsqrtf(rr), -1.0f) : 0.0f;
    }
}

// Cell of a position: (x - left) / cell_size truncated through a signed 64-bit
// integer and kept to 32 bits, as the reference's `integer c = expr;` does on
// x86-64 (MPS_CAL_expl_v1.0/MPS_GPU.cpp:263-266).  Returns g.ncells (the
// sentinel that sorts last) when the particle is outside the grid.
__device__ __forceinline__ uint32_t cell_of_pos(const Grid& g, float x, float y, float z, bool* nan_flag) {
    if (!(x == x) || !(y == y) || !(z == z)) {
        *nan_flag = true;
        return g.ncells;
    }
    uint32_t cx = (uint32_t)(long long)__fdiv_rn(__fsub_rn(x, g.left), g.cell_size);
    uint32_t cy = (uint32_t)(long long)__fdiv_rn(__fsub_rn(y, g.back), g.cell_yz);
    uint32_t cz = (uint32_t)(long long)__fdiv_rn(__fsub_rn(z, g.bottom), g.cell_yz);
    if (cx >= g.cdx || cy >= g.cdy || cz >= g.cdz) return g.ncells;
    return cz * g.sheet + cy * g.cdx + cx;
}

// The particles of the reference's 27 linked cells (MPS_GPU::makeLink,
// MPS_CAL_expl_v1.0/MPS_GPU.cpp:168-243) as 9 rows (3 in 2D): row (dz, dy)
// covers cells c0-1, c0, c0+1 with c0 = c + dz*sheet + dy*cdx, each kept when
// its id (with unsigned wrap) is below ncells, exactly the reference's test.
// The kept cells are consecutive, so their particles are one index range;
// rows come in the reference's order, so visiting rows in order and indices
// ascending reproduces the reference's summation order.  On a grid with
// reach 2 the rows run over dz, dy in [-2, 2] in the same order (25 rows),
// and the candidates still come in ascending index order.
struct RowRange { uint32_t lo, hi; };

__device__ __forceinline__ void row_offsets(const Grid& g, int row, int* dz, int* dy) {
    const int w = 2 * g.reach + 1;
    if (g.dim == 3) { *dz = row / w - g.reach; *dy = row % w - g.reach; }
    else { *dz = 0; *dy = row - g.reach; }
}

__device__ __forceinline__ RowRange link_row(const Grid& g, const uint32_t* __restrict__ cell_start, uint32_t c,
                                             int row) {
    int dz, dy;
    row_offsets(g, row, &dz, &dy);
    uint32_t c0 = c + (uint32_t)dz * g.sheet + (uint32_t)dy * g.cdx;
    uint32_t a = c0 - 1u, b = c0 + 1u;
    bool va = a < g.ncells, v0 = c0 < g.ncells, vb = b < g.ncells;
    RowRange r{0u, 0u};
    uint32_t first, last;
    if (va) first = a; else if (v0) first = c0; else if (vb) first = b; else return r;
    if (vb) last = b; else if (v0) last = c0; else last = a;
    r.lo = __ldg(cell_start + first);
    r.hi = __ldg(cell_start + last + 1u);
    return r;
}

__device__ __forceinline__ int link_rows(const Grid& g) {
    const int w = 2 * g.reach + 1;
    return g.dim == 3 ? w * w : w;
}

// Culling of the linked cells: the distances from a particle to the faces of
// its own cell bound the distance to any particle of a neighbouring cell.  A
// row (or its first or last cell) farther than re plus a margin cannot hold
// a particle that passes a stage's distance test, so leaving it out removes
// only candidates that contribute nothing: the remaining candidates keep the
// reference's order and every sum is unchanged.  The margin (1e-4 of a cell)
// covers the rounding of the cell assignment and of the face positions.
struct CellNear {
    float xl, xr, yl, yr, zl, zr;  // to the low / high face along each axis
    float re2;                     // (re + margin)^2
    float hyz;                     // cell edge along y and z (rows beyond the first)
};

__device__ __forceinline__ CellNear cell_near(const Grid& g, uint32_t c, float x, float y, float z, float re) {
    const uint32_t cz = c / g.sheet, rem = c - cz * g.sheet;
    const uint32_t cy = rem / g.cdx, cx = rem - cy * g.cdx;
    const float x0 = g.left + g.cell_size * (float)cx;
    const float y0 = g.back + g.cell_yz * (float)cy;
    const float z0 = g.bottom + g.cell_yz * (float)cz;
    CellNear n;
    n.xl = fmaxf(x - x0, 0.f);
    n.xr = fmaxf(x0 + g.cell_size - x, 0.f);
    n.yl = fmaxf(y - y0, 0.f);
    n.yr = fmaxf(y0 + g.cell_yz - y, 0.f);
    n.zl = fmaxf(z - z0, 0.f);
    n.zr = fmaxf(z0 + g.cell_yz - z, 0.f);
    const float r = re + 1e-4f * g.cell_size;
    n.re2 = r * r;
    n.hyz = g.cell_yz;
    return n;
}

// link_row restricted to the cells that can hold a particle within re
// row (dz, dy) of the walk
__device__ __forceinline__ RowRange link_row_near_at(const Grid& g, const uint32_t* __restrict__ cell_start,
                                                     uint32_t c, int dz, int dy, const CellNear& n) {
    // distance to the row: the face of the own cell plus the whole cells between
    float d2 = 0.f;
    if (dy < 0) { const float t = fmaf(n.hyz, (float)(-dy - 1), n.yl); d2 += t * t; }
    else if (dy > 0) { const float t = fmaf(n.hyz, (float)(dy - 1), n.yr); d2 += t * t; }
    if (dz < 0) { const float t = fmaf(n.hyz, (float)(-dz - 1), n.zl); d2 += t * t; }
    else if (dz > 0) { const float t = fmaf(n.hyz, (float)(dz - 1), n.zr); d2 += t * t; }
    RowRange r{0u, 0u};
    if (d2 >= n.re2) return r;
    const bool wa = d2 + n.xl * n.xl < n.re2, wb = d2 + n.xr * n.xr < n.re2;
    const uint32_t c0 = c + (uint32_t)dz * g.sheet + (uint32_t)dy * g.cdx;
    const uint32_t a = c0 - 1u, b = c0 + 1u;
    const bool va = wa && a < g.ncells, v0 = c0 < g.ncells, vb = wb && b < g.ncells;
    uint32_t first, last;
    if (va) first = a; else if (v0) first = c0; else if (vb) first = b; else return r;
    if (vb) last = b; else if (v0) last = c0; else last = a;
    r.lo = __ldg(cell_start + first);
    r.hi = __ldg(cell_start + last + 1u);
    return r;
}

__device__ __forceinline__ RowRange link_row_near(const Grid& g, const uint32_t* __restrict__ cell_start, uint32_t c,
                                                  int row, const CellNear& n) {
    int dz, dy;
    row_offsets(g, row, &dz, &dy);
    return link_row_near_at(g, cell_start, c, dz, dy, n);
}

// link_row_near on the reference's grid (reach 1): row r of 9 (3 in 2D)
__device__ __forceinline__ RowRange link_row_near_ref(const Grid& g, const uint32_t* __restrict__ cell_start,
                                                      uint32_t c, int row, const CellNear& n) {
    int dz, dy;
    if (g.dim == 3) { dz = row / 3 - 1; dy = row % 3 - 1; }
    else { dz = 0; dy = row - 1; }
    float d2 = 0.f;
    if (dy < 0) d2 += n.yl * n.yl;
    else if (dy > 0) d2 += n.yr * n.yr;
    if (dz < 0) d2 += n.zl * n.zl;
    else if (dz > 0) d2 += n.zr * n.zr;
    RowRange r{0u, 0u};
    if (d2 >= n.re2) return r;
    const bool wa = d2 + n.xl * n.xl < n.re2, wb = d2 + n.xr * n.xr < n.re2;
    const uint32_t c0 = c + (uint32_t)dz * g.sheet + (uint32_t)dy * g.cdx;
    const uint32_t a = c0 - 1u, b = c0 + 1u;
    const bool va = wa && a < g.ncells, v0 = c0 < g.ncells, vb = wb && b < g.ncells;
    uint32_t first, last;
    if (va) first = a; else if (v0) first = c0; else if (vb) first = b; else return r;
    if (vb) last = b; else if (v0) last = c0; else last = a;
    r.lo = __ldg(cell_start + first);
    r.hi = __ldg(cell_start + last + 1u);
    return r;
}

// A warp's walk over all its rows as one list of candidates.  Lane r looks
// up row r (link_row_near; at most 25 rows, so one lookup per lane, all in
// parallel), an inclusive scan of the row lengths numbers the candidates of
// all rows in walk order (rows in order, indices ascending within a row),
// and candidate f of that numbering is fetched with a 5-step search over the
// lanes' row ends.  Every 32 consecutive candidates fill one batch of the
// warp, whichever rows they come from, in the same order as the row-by-row
// walk: ordered sums over the batches add the same terms in the same order.
struct FlatWalk {
    uint32_t total;  // candidates over all rows
    uint32_t end;    // this lane's row: one past its last candidate in walk order (total past the rows)
    int base;        // this lane's row: particle index minus walk position
};

__device__ __forceinline__ FlatWalk flat_walk_of(RowRange rg, uint32_t lane) {
    const uint32_t len = rg.hi - rg.lo;
    uint32_t e = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, e, o);
        if ((int)lane >= o) e += t;
    }
    FlatWalk w;
    w.total = __shfl_sync(0xffffffffu, e, 31);
    w.end = e;
    w.base = (int)rg.lo - (int)(e - len);
    return w;
}

__device__ __forceinline__ FlatWalk flat_walk(const Grid& g, const uint32_t* __restrict__ cell_start, uint32_t c,
                                              const CellNear& n, uint32_t lane) {
    RowRange rg{0u, 0u};
    if ((int)lane < link_rows(g)) rg = link_row_near(g, cell_start, c, (int)lane, n);
    return flat_walk_of(rg, lane);
}

// the particle index of candidate f (f < total; every lane calls it)
__device__ __forceinline__ uint32_t flat_at(const FlatWalk& w, uint32_t f) {
    int r = 0;
#pragma unroll
    for (int step = 16; step > 0; step >>= 1) {
        const uint32_t e = __shfl_sync(0xffffffffu, w.end, r + step - 1);
        if (e <= f) r += step;
    }
    return (uint32_t)((int)f + __shfl_sync(0xffffffffu, w.base, r));
}

// body(j, in) for each batch of 32 candidates of a warp's walk, in walk
// order (lane L gets the batch's L-th candidate; `in` is false past the
// end).  FLAT walks the rows as one list (flat_walk: the rows' lookups in
// parallel, full batches) on any grid; the other form walks the reference's
// grid (reach 1) row by row.  Both visit the same candidates in the same
// order.  The flat form pays on the refined grid (up to 25 short rows); on
// the reference's grid (9 rows of about 200 candidates) the row form is as
// fast and is what the exact kernels use: exact arithmetic keeps the
// reference's grid (the refined one is built for fast arithmetic only).
template <bool FLAT, class F>
__device__ __forceinline__ void walk_cells(const Grid& g, const uint32_t* __restrict__ cs, uint32_t c,
                                           const CellNear& nr, uint32_t lane, F&& body) {
    if (FLAT) {
        const FlatWalk fw = flat_walk(g, cs, c, nr, lane);
        for (uint32_t f0 = 0; f0 < fw.total; f0 += 32) {
            const bool in = f0 + lane < fw.total;
            body(flat_at(fw, in ? f0 + lane : fw.total - 1), in);
        }
    } else {
        const int rows = g.dim == 3 ? 9 : 3;
        for (int row = 0; row < rows; row++) {
            const RowRange rg = link_row_near_ref(g, cs, c, row, nr);
            for (uint32_t base = rg.lo; base < rg.hi; base += 32) body(base + lane, base + lane < rg.hi);
        }
    }
}

}  // namespace mpsb
