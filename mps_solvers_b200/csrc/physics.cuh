// physics.cuh -- launchers of the particle-stage kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "cellsort.cuh"
#include "mps_device.cuh"

namespace mpsb {

// A fluid-list entry that holds no particle (it pads each gather warp's run
// of fluid particles to an even length)
constexpr uint32_t LIST_GAP = 0xffffffffu;

// Particle state in one buffer set (sorted order).
struct State {
    float4* pos;      // x y z, w = type bits
    float4* vel;      // u v w, w unused (0)
    float* press;
    float* n;
    uint32_t* id;     // GEO.dat index
    uint32_t* cell;   // cell id from the last rebuild (i_cell_list)
};

struct StageArgs {
    State cur;                 // current state
    const uint32_t* cell_start;  // ncells + 1 entries
    float4* tmp;               // pending update (one float4 per particle)
    Scalars* sc;
    Grid g;
    Phys P;
    bool exact;
    int semi;                  // semi-implicit (v4.0) rules
    // compact particle lists from the last rebuild (nullptr: all particles);
    // the fluid list holds LIST_GAP entries (see gather_tail), cap_fluid
    // counts them
    const uint32_t* list_fluid = nullptr;
    const uint32_t* n_fluid = nullptr;
    uint32_t cap_fluid = 0;
    const uint32_t* list_solid = nullptr;  // fluid + wall (type != 2)
    const uint32_t* n_solid = nullptr;
    uint32_t cap_solid = 0;
    BatchDev batch;            // scenes of a batch (n == 0: one scene, g and P)
    int threads = 256;         // block size of the particle-stage kernels (autotuned: 64, 128, 256)
};

// Scene-local view of particle i: its scene, its grid, its cell table (the
// global table from the grid's first cell) and its cell in that grid.
struct Local {
    Grid g;
    const uint32_t* cs;
    uint32_t c;
    uint32_t s;
};

// BT: the launch belongs to a batch (a.batch.n > 0), decided on the host so
// that a single scene's kernels carry no batch code.
template <bool BT>
__device__ __forceinline__ Local local_of(const StageArgs& a, uint32_t i) {
    Local L;
    const uint32_t cell = a.cur.cell[i];
    if (BT) {
        L.s = __ldg(a.batch.sid_of_id + a.cur.id[i]);
        L.g = a.batch.grid[L.s];
        L.cs = a.cell_start + L.g.base;
        L.c = cell - L.g.base;
    } else {
        L.s = 0;
        L.g = a.g;
        L.cs = a.cell_start;
        L.c = cell;
    }
    return L;
}

template <bool BT>
__device__ __forceinline__ Phys phys_of(const StageArgs& a, uint32_t s) {
    if (BT) return a.batch.phys[s];
    return a.P;
}
template <bool BT>
__device__ __forceinline__ float dt_of(const StageArgs& a, uint32_t s) {
    return BT ? a.batch.dt[s] : a.sc->dt;
}

// the same, decided per launch on the device (set-up kernels)
__device__ __forceinline__ Local local_of(const StageArgs& a, uint32_t i) {
    return a.batch.n ? local_of<true>(a, i) : local_of<false>(a, i);
}
__device__ __forceinline__ Phys phys_of(const StageArgs& a, uint32_t s) {
    return a.batch.n ? phys_of<true>(a, s) : phys_of<false>(a, s);
}

// the merge rebuild's reorder (cellsort.cuh: launch_merge_keys_sort first):
// every particle moved to its merged position with the pending update
// applied, and the new cell table cs_new from cs_old
void launch_merge_gather(const State& src, const State& dst, const MergeScratch& m, const uint32_t* cs_old,
                         uint32_t* cs_new, uint32_t ncells, const float4* tmp, int apply, uint32_t* index_of_id,
                         Scalars* sc, uint32_t cap, cudaStream_t st, uint32_t* list_fluid, uint32_t* list_solid,
                         const BatchDev& batch);

// reorder after a sort: dst[p] = src[perm[p]] with the pending update applied
void launch_gather(const State& src, const State& dst, const uint32_t* perm, const uint32_t* keys_sorted,
                   const float4* tmp, int apply, uint32_t* index_of_id, Scalars* sc, uint32_t cap, cudaStream_t st,
                   uint32_t* list_fluid, uint32_t* list_solid, const BatchDev& batch, uint32_t* cell_start,
                   uint32_t ncells);

// update_dt: max |u|^2, then dt on the device
void launch_update_dt(const StageArgs& a, uint32_t cap, cudaStream_t st);
// stage kernels
void launch_visc(const StageArgs& a, uint32_t cap, cudaStream_t st);
void launch_collision(const StageArgs& a, uint32_t cap, cudaStream_t st);
void launch_pnd(const StageArgs& a, int eos, int all_types, uint32_t cap, cudaStream_t st);
void launch_dummy_press(const StageArgs& a, const uint32_t* normal_id_of, const uint32_t* index_of_id, uint32_t cap,
                        cudaStream_t st);
void launch_dash(const StageArgs& a, uint32_t cap, cudaStream_t st);
void launch_step_end(Scalars* sc, const BatchDev& batch, cudaStream_t st);

// host-layout staging (x y z per particle) <-> the float4 state
struct Staging {
    float* pos3;
    float* vel3;
    float* press;
    float* n;
    uint32_t* id;
    uint32_t* type;
};
// sorted order (by_id = 0) or by GEO index into np0 entries (by_id = 1)
void launch_unpack(const State& s, const Staging& out, int by_id, uint32_t np0, const Scalars* sc, uint32_t cap,
                   cudaStream_t st);
// overwrite the selected fields of the active particles (mask bits: 1 pos,
// 2 vel, 4 press, 8 n)
void launch_pack(const State& s, const Staging& in, int mask, const Scalars* sc, uint32_t cap, cudaStream_t st);

// initialisation
// n0 and the particle it belongs to: max n with the lowest index on ties
void launch_nzero(const float* n, Scalars* sc, unsigned long long* best, uint32_t cap, cudaStream_t st);
// the same over the particle range [lo, hi) (one scene of a batch)
void launch_nzero_range(const float* n, uint32_t lo, uint32_t hi, unsigned long long* best, cudaStream_t st);
// lambda = sum over j of r^2 w(r0) around particle `best`, in index order
void launch_lambda(const StageArgs& a, const unsigned long long* best, float* lambda_out, cudaStream_t st);
// nearest type-1 particle (first in index order) within sqrt(2) r0 of each
// type-2 particle, stored by GEO.dat index
void launch_normals(const StageArgs& a, int reach, int reach_yz, uint32_t* normal_id_of, uint32_t cap,
                    cudaStream_t st);

// Prescribed rigid motions of boundary particles (the reference's
// MOTION::doMotion hook).  Motion m moves its particles to
// x0 + vel tau + amp (sin(omega tau + phase) - sin(phase)) with velocity
// vel + amp omega cos(omega tau + phase), tau = time - t0 (double, rounded
// once to float), at the start of every step.
constexpr int MPS_MAX_MOTIONS = 8;
constexpr uint32_t NO_MOTION = 0xFFFFFFFFu;
struct MotionSet {
    int n = 0;
    double t0[MPS_MAX_MOTIONS], vel[MPS_MAX_MOTIONS][3], amp[MPS_MAX_MOTIONS][3], omega[MPS_MAX_MOTIONS],
        phase[MPS_MAX_MOTIONS];
};
// give motion m to the wall and dummy particles inside [lo, hi] that have
// none (motion_of and x0 are indexed by GEO.dat id); adds the count to *count
void launch_motion_select(const State& s, const Scalars* sc, const float lo[3], const float hi[3], uint32_t m,
                          uint32_t* motion_of, float4* x0, uint32_t* count, uint32_t cap, cudaStream_t st);
// set the velocity of every particle with a motion to zero
void launch_motion_stop(const State& s, const Scalars* sc, const uint32_t* motion_of, uint32_t cap, cudaStream_t st);
// place the moving particles for the step starting at sc->time
void launch_motion(const State& s, const Scalars* sc, const uint32_t* motion_of, const float4* x0,
                   const MotionSet& M, uint32_t cap, cudaStream_t st);

}  // namespace mpsb
