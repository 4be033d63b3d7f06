// mps_device.cuh -- device-side types and helpers shared by the kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace mpsb {

// Cell grid of the reference's cell list (MPS_CAL_expl_v1.0/MPS.cpp:567-642).
struct Grid {
    float left, back, bottom, cell_size;
    uint32_t cdx, cdy, cdz, sheet, ncells;
    int dim;
    uint32_t base;  // first global cell id of this grid (scenes of a batch; 0 otherwise)
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
    uint32_t cy = (uint32_t)(long long)__fdiv_rn(__fsub_rn(y, g.back), g.cell_size);
    uint32_t cz = (uint32_t)(long long)__fdiv_rn(__fsub_rn(z, g.bottom), g.cell_size);
    if (cx >= g.cdx || cy >= g.cdy || cz >= g.cdz) return g.ncells;
    return cz * g.sheet + cy * g.cdx + cx;
}

// The particles of the reference's 27 linked cells (MPS_GPU::makeLink,
// MPS_CAL_expl_v1.0/MPS_GPU.cpp:168-243) as 9 rows (3 in 2D): row (dz, dy)
// covers cells c0-1, c0, c0+1 with c0 = c + dz*sheet + dy*cdx, each kept when
// its id (with unsigned wrap) is below ncells, exactly the reference's test.
// The kept cells are consecutive, so their particles are one index range;
// rows come in the reference's order, so visiting rows in order and indices
// ascending reproduces the reference's summation order.
struct RowRange { uint32_t lo, hi; };

__device__ __forceinline__ RowRange link_row(const Grid& g, const uint32_t* __restrict__ cell_start, uint32_t c,
                                             int row) {
    int dz, dy;
    if (g.dim == 3) { dz = row / 3 - 1; dy = row % 3 - 1; }
    else { dz = 0; dy = row - 1; }
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

__device__ __forceinline__ int link_rows(const Grid& g) { return g.dim == 3 ? 9 : 3; }

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
};

__device__ __forceinline__ CellNear cell_near(const Grid& g, uint32_t c, float x, float y, float z, float re) {
    const uint32_t cz = c / g.sheet, rem = c - cz * g.sheet;
    const uint32_t cy = rem / g.cdx, cx = rem - cy * g.cdx;
    const float x0 = g.left + g.cell_size * (float)cx;
    const float y0 = g.back + g.cell_size * (float)cy;
    const float z0 = g.bottom + g.cell_size * (float)cz;
    CellNear n;
    n.xl = fmaxf(x - x0, 0.f);
    n.xr = fmaxf(x0 + g.cell_size - x, 0.f);
    n.yl = fmaxf(y - y0, 0.f);
    n.yr = fmaxf(y0 + g.cell_size - y, 0.f);
    n.zl = fmaxf(z - z0, 0.f);
    n.zr = fmaxf(z0 + g.cell_size - z, 0.f);
    const float r = re + 1e-4f * g.cell_size;
    n.re2 = r * r;
    return n;
}

// link_row restricted to the cells that can hold a particle within re
__device__ __forceinline__ RowRange link_row_near(const Grid& g, const uint32_t* __restrict__ cell_start, uint32_t c,
                                                  int row, const CellNear& n) {
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

}  // namespace mpsb
