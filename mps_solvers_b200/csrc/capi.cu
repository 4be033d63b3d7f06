// capi.cu -- libmps_b200.so: the C ABI of include/mps_capi.h.
//
// A handle owns one scene on one device: two particle buffer sets (the
// rebuild gathers from one into the other), the sort scratch, the cell
// table, the per-step device scalars, and one stream.  Every step is the
// reference's stage order; with use_graph the launches of a step are
// captured once per buffer parity and replayed.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstddef>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mps_capi.h"
#include "cellsort.cuh"
#include "host_io.h"
#include "physics.cuh"
#include "ppe.cuh"
#include "surface.cuh"

using namespace mpsb;

struct mps_handle {
    int dev = 0;
    cudaStream_t stream = nullptr;
    mps_options opt{};
    mps_params prm{};
    HostGrid hg{};
    HostConst hc{};
    Grid g{};
    Phys P{};
    uint32_t np0 = 0, nb2 = 0, nb1 = 0, cap = 0;
    int passes = 1;
    int normal_reach = 1, normal_reach_yz = 1;
    // device memory
    State S[2]{};
    int cur = 0;
    float4* tmp = nullptr;
    uint32_t* index_of_id = nullptr;
    uint32_t* normal_id_of = nullptr;
    uint32_t* cell_tab[2] = {nullptr, nullptr};  // cell table of each state buffer's order
    MergeScratch merge{};   // the merge rebuild's scratch (options.rebuild_merge)
    bool merge_ready = false;
    bool sorted = false;    // the current state buffer is sorted and its cell table valid
    uint32_t moving = 0;    // wall and dummy particles with a motion
    uint32_t* list_fluid = nullptr;
    uint32_t* list_solid = nullptr;
    uint32_t cap_fluid = 0, cap_solid = 0;
    uint32_t cap_flist = 1;  // fluid list entries: the fluid and a gap per gather warp at most
    SortScratch sort{};
    Scalars* sc = nullptr;
    unsigned long long* best = nullptr;
    float* lambda_dev = nullptr;
    PpeWork ppe{};
    PpeWork cn{};  // Crank-Nicolson viscosity system (options.visc_implicit)
    Staging stage{};
    // graphs, one per buffer parity
    // one graph per buffer parity, and for the learned compact preconditioner
    // per kind of step (index parity + 2 when the step evaluates the network)
    cudaGraphExec_t graph[4] = {nullptr, nullptr, nullptr, nullptr};
    int pending_apply = APPLY_NONE;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // per-stage profiling: events recorded between stages when enabled
    bool prof_on = false;
    std::vector<cudaEvent_t> prof_ev;
    std::vector<int> prof_tag;
    size_t prof_used = 0;
    int launches = 0;  // kernels enqueued by the last enqueue_step
    cudaError_t launch_err = cudaSuccess;  // first failed launch not seen by cudaGetLastError
    std::string err;
    std::vector<void*> allocs;
    // batch of scenes (nscenes == 0: a single scene)
    uint32_t nscenes = 0;
    BatchDev batch{};
    std::vector<uint32_t> id_base;   // first particle id of each scene, then the total
    std::vector<uint32_t> scene_nb2, scene_nb1;
    std::vector<Phys> scene_phys;
    std::vector<Grid> scene_grid;
    std::vector<HostConst> scene_hc;
    Phys* phys_dev = nullptr;
    bool graph_off = false;          // stream capture refused: direct launches
    std::string graph_note;
    int stage_threads = 256;         // block size of the particle-stage kernels (autotuned)
    SurfaceWork surf;                // marching-cubes free surface
    // prescribed boundary motions (allocated by the first mps_add_wall_motion)
    MotionSet mot{};
    uint32_t* motion_of = nullptr;   // per GEO.dat id
    float4* motion_x0 = nullptr;     // per GEO.dat id
    uint32_t* motion_count = nullptr;
    // the device scalars as the last read_status saw them; valid until work
    // that may change the particle count is enqueued (steps, rebuilds)
    bool sc_valid = false;
    Scalars sc_host{};
};

static void drop_graphs(mps_handle* h);

// ---------------------------------------------------------------- helpers
static const char* kStatusNames[] = {"ok",
                                     "io error",
                                     "cells too thin",
                                     "dt too small",
                                     "particle outside the grid",
                                     "CG did not converge",
                                     "device wait timed out",
                                     "CUDA error",
                                     "NaN detected",
                                     "invalid argument",
                                     "capacity exceeded"};

extern "C" const char* mps_status_string(mps_status s) {
    int k = (int)s;
    if (k < 0 || k > 10) return "unknown";
    return kStatusNames[k];
}

#define CK(call)                                                                 \
    do {                                                                         \
        cudaError_t _e = (call);                                                 \
        if (_e != cudaSuccess) {                                                 \
            h->err = std::string(#call) + ": " + cudaGetErrorString(_e);         \
            return MPS_ERR_CUDA;                                                 \
        }                                                                        \
    } while (0)

template <class T>
static cudaError_t dalloc(mps_handle* h, T** p, size_t count) {
    void* v = nullptr;
    cudaError_t e = cudaMalloc(&v, count * sizeof(T) + 16);
    if (e == cudaSuccess) {
        h->allocs.push_back(v);
        cudaMemsetAsync(v, 0, count * sizeof(T) + 16, h->stream);
    }
    *p = (T*)v;
    return e;
}

static StageArgs stage_args(mps_handle* h) {
    StageArgs a;
    a.cur = h->S[h->cur];
    a.cell_start = h->cell_tab[h->cur];
    a.tmp = h->tmp;
    a.sc = h->sc;
    a.g = h->g;
    a.P = h->P;
    a.exact = h->opt.arith == MPS_ARITH_EXACT;
    a.semi = h->opt.method == MPS_METHOD_SEMI_IMPLICIT;
    a.list_fluid = h->list_fluid;
    a.n_fluid = &h->sc->n_fluid;
    a.cap_fluid = h->cap_flist;
    a.list_solid = h->list_solid;
    a.n_solid = &h->sc->n_solid;
    a.cap_solid = h->cap_solid;
    a.batch = h->batch;
    a.threads = h->stage_threads;
    return a;
}

// Stage tags of mps_profile_steps (names in kStageNames).
enum { ST_UPDATE_DT = 0, ST_VISC, ST_COLLISION, ST_PND, ST_PRESSURE, ST_DASH, ST_STEP_END, ST_KEYS, ST_SORT,
       ST_CELLS, ST_GATHER, ST_PPE_SOLVE, ST_MOTION, ST_COUNT };
static const char* kStageNames[ST_COUNT] = {"update_dt", "visc",       "collision",  "pnd",
                                            "pressure",  "dash",       "step_end",   "cell_keys",
                                            "radix_sort", "cell_table", "gather",     "ppe_solve",
                                            "motion"};

static void mark(mps_handle* h, int tag) {
    if (!h->prof_on) return;
    if (h->prof_used == h->prof_ev.size()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        h->prof_ev.push_back(e);
        h->prof_tag.push_back(0);
    }
    h->prof_tag[h->prof_used] = tag;
    cudaEventRecord(h->prof_ev[h->prof_used], h->stream);
    h->prof_used++;
}

// The reference's divideCell: keys (after the pending update), stable sort,
// cell table, gather into the other buffer set.
// The merge rebuild (cellsort.cuh) when at most MERGE_SMEM_CAP particles can
// change cell between two rebuilds (fluid and moving walls) and the current
// order is a sorted one; else the full radix sort.  Both give the same order.
// The compact PPE layout on or off; with the learned preconditioner the
// compact solver applies S' by compact columns (the 8-byte solver by
// particle columns).
static void set_compact(mps_handle* h, bool on) {
    h->ppe.c16 = on && h->ppe.c16_ready;
    h->ppe.c16_learned = h->ppe.c16 && h->opt.precond == MPS_PRECOND_LEARNED && h->ppe.sp_ent != nullptr &&
                         h->ppe.cr2 != nullptr;
}

static bool use_merge(const mps_handle* h) {
    return h->merge_ready && h->sorted && (uint64_t)h->cap_fluid + h->moving <= MERGE_SMEM_CAP;
}

static void rebuild(mps_handle* h, int apply) {
    h->sc_valid = false;
    cudaStream_t st = h->stream;
    State& src = h->S[h->cur];
    State& dst = h->S[h->cur ^ 1];
    uint32_t* cs_new = h->cell_tab[h->cur ^ 1];
    if (use_merge(h)) {
        mark(h, ST_SORT);
        launch_merge_keys_sort(src.pos, h->tmp, apply, h->g, h->sc, src.id, h->batch, src.cell, h->merge, h->cap, st);
        mark(h, ST_GATHER);  // the merge gather also derives the cell table
        launch_merge_gather(src, dst, h->merge, h->cell_tab[h->cur], cs_new, h->g.ncells, h->tmp, apply,
                            h->index_of_id, h->sc, h->cap, st, h->list_fluid, h->list_solid, h->batch);
        h->launches += 3;
    } else {
        mark(h, ST_SORT);  // the keys are computed by the first pass's upsweep
        const int r =
            launch_keys_and_sort(src.pos, h->tmp, apply, h->g, h->sc, src.id, h->batch, h->sort, h->passes, st);
        mark(h, ST_GATHER);  // the gather also fills the cell table
        launch_gather(src, dst, h->sort.vals[r], h->sort.keys[r], h->tmp, apply, h->index_of_id, h->sc, h->cap, st,
                      h->list_fluid, h->list_solid, h->batch, cs_new, h->g.ncells);
        h->launches += 1 + h->passes * (h->sort.tiles > SORT_FUSED_SCAN_TILES ? 3 : 2);
    }
    h->cur ^= 1;
    h->sorted = true;
}

// One step in the reference's order.
//  explicit: MPS_GPU_EXPL::step (MPS_CAL_expl_v1.0/MPS_GPU_EXPL.cpp:277-339)
//  semi:     MPS_CPU_EXPL::step (MPS_CAL_v4.0/MPS_CPU_EXPL.cpp:79-135)
static void enqueue_step(mps_handle* h) {
    h->sc_valid = false;
    cudaStream_t st = h->stream;
    const uint32_t cap = h->cap;
    h->launches = 0;
    if (h->mot.n) {  // the reference's motion(); divideCell(); at the top of a step
        mark(h, ST_MOTION);
        launch_motion(h->S[h->cur], h->sc, h->motion_of, h->motion_x0, h->mot, cap, st);
        rebuild(h, APPLY_NONE);
        h->launches += 1;
    }
    mark(h, ST_UPDATE_DT);
    launch_update_dt(stage_args(h), cap, st);
    mark(h, ST_VISC);
    if (h->cn.ready) {  // MPS_CPU_IMPL::visCrankNicolson: x, y, z in turn, then divideCell
        for (int c = 0; c < (int)h->g.dim; c++) {
            h->launches += ppe_enqueue_cn(h->cn, stage_args(h), h->opt, c, h->ppe.n0_64, h->ppe.lambda64, cap, st);
            if (h->cn.launch_err != cudaSuccess) h->launch_err = h->cn.launch_err;
        }
        rebuild(h, APPLY_NONE);
    } else {
        launch_visc(stage_args(h), cap, st);
        rebuild(h, APPLY_SET_VEL);
    }
    mark(h, ST_COLLISION);
    launch_collision(stage_args(h), cap, st);
    rebuild(h, APPLY_ADD_VEL);
    mark(h, ST_PND);
    if (h->opt.method == MPS_METHOD_EXPLICIT) {
        launch_pnd(stage_args(h), 1, 0, cap, st);
        mark(h, ST_PRESSURE);
        launch_dummy_press(stage_args(h), h->normal_id_of, h->index_of_id, cap, st);
        h->launches += 2;
    } else {
        launch_pnd(stage_args(h), 0, 0, cap, st);
        mark(h, ST_PRESSURE);
        h->launches += 1 + ppe_enqueue_setup(h->ppe, stage_args(h), h->opt, cap, st);
        mark(h, ST_PPE_SOLVE);
        h->launches += ppe_enqueue_solve(h->ppe, stage_args(h), h->opt, cap, st);
        if (h->ppe.launch_err != cudaSuccess) h->launch_err = h->ppe.launch_err;
    }
    mark(h, ST_DASH);
    launch_dash(stage_args(h), cap, st);
    rebuild(h, APPLY_ADD_VEL);
    mark(h, ST_STEP_END);
    if (h->opt.method == MPS_METHOD_SEMI_IMPLICIT) {
        launch_update_dt(stage_args(h), cap, st);
        h->launches += 1;
    }
    launch_step_end(h->sc, h->batch, st);
    h->launches += 5;
}

static mps_status read_status(mps_handle* h, Scalars* out) {
    Scalars s;
    CK(cudaMemcpyAsync(&s, h->sc, sizeof(Scalars), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->sc_host = s;
    h->sc_valid = true;
    if (out) *out = s;
    if (s.err & ERR_NAN) { h->err = "NaN in particle state"; return MPS_ERR_NAN; }
    if (s.err & ERR_DT_TOO_SMALL) { h->err = "dt below dt_min"; return MPS_ERR_DT_TOO_SMALL; }
    if (s.err & ERR_DEVICE_TIMEOUT) { h->err = "device wait timed out"; return MPS_ERR_DEVICE_TIMEOUT; }
    if (s.err & ERR_CG_NOT_CONVERGED) { h->err = "PPE CG did not reach its tolerance"; return MPS_ERR_CG_NOT_CONVERGED; }
    if (s.err & ERR_PARTICLE_OUT) { h->err = "particle left the grid"; return MPS_ERR_PARTICLE_OUT; }
    if (s.err & ERR_CAPACITY) { h->err = "a particle has more PPE neighbours than the matrix stride holds"; return MPS_ERR_CAPACITY; }
    return MPS_OK;
}

// ---------------------------------------------------------------- create
extern "C" void mps_default_options(mps_options* o) {
    memset(o, 0, sizeof *o);
    o->method = MPS_METHOD_EXPLICIT;
    o->arith = MPS_ARITH_EXACT;
    o->device = 0;
    o->use_graph = 1;
    o->cg_tol = 1e-8;
    o->cg_max_iter = 10000;
    o->cg_check_every = 1000;
    o->cg_inner_digits = 4;
    o->precond = MPS_PRECOND_DIAGONAL;
    o->capacity = 0;
}

// constants of a scene that do not depend on n0
static Phys base_phys(const mps_params& prm) {
    Phys P;
    memset(&P, 0, sizeof P);
    P.rzero = prm.rzero;
    P.rlap = prm.rlap;
    P.col_dis = prm.col_dis;
    P.col_rate = prm.col_rate;
    P.niu = prm.niu;
    P.rho = prm.rho;
    P.dt_max = prm.dt_max;
    P.dt_min = prm.dt_min;
    P.cfl_dp = prm.cfl * prm.dp;
    P.beta = prm.beta;
    P.g[0] = 0.0f;
    P.g[1] = 0.0f;
    P.g[2] = -9.81f;
    P.dim_f = (float)prm.dim;
    P.rzero_thr = rr_threshold(prm.rzero);
    P.rlap_thr = rr_threshold(prm.rlap);
    P.col_thr = rr_threshold(prm.col_dis);
    P.rzero2 = prm.rzero * prm.rzero;
    return P;
}

// MPS_CPU::Initial / MPS::calOnce of MPS_CAL_v4.0 (MPS_CPU.cpp:54-122,
// MPS.cpp:305-370): the constants from n0 and lambda in double
static HostConst semi_constants(const mps_params& prm, double n0, double lambda) {
    HostConst c;
    c.nzero = (float)n0;
    c.lambda = (float)lambda;
    c.alpha = (float)(1.0 / ((double)prm.rho * prm.cs * prm.cs));
    c.one_over_alpha = (float)((double)prm.rho * prm.cs * prm.cs);
    c.one_over_rho = (float)(1.0 / (double)prm.rho);
    c.one_over_nzero = (float)(1.0 / n0);
    c.one_over_dim = (float)(1.0 / (double)prm.dim);
    c.one_over_dt = (float)(1.0 / (double)prm.dt_max);
    c.c_lap = (float)((2.0 * prm.dim) / (n0 * lambda));
    return c;
}

static void apply_constants(Phys& P, const HostConst& c) {
    P.nzero = c.nzero;
    P.one_over_nzero = c.one_over_nzero;
    P.one_over_alpha = c.one_over_alpha;
    P.one_over_rho = c.one_over_rho;
    P.c_lap = c.c_lap;
    P.lambda = c.lambda;
    P.alpha = c.alpha;
    P.one_over_dt_fixed = c.one_over_dt;
}

// The merge rebuild's scratch, unless the options turn it off or more
// particles can move than its one-block sort takes (use_merge).
static cudaError_t merge_setup(mps_handle* h) {
    if (h->opt.rebuild_merge != 0 || (uint64_t)h->cap_fluid > MERGE_SMEM_CAP) return cudaSuccess;
    size_t p2 = 1;  // the sort's global-memory case pads to a power of two
    while (p2 < h->cap) p2 <<= 1;
    cudaError_t e;
    if ((e = dalloc(h, &h->merge.newkey, h->cap)) != cudaSuccess) return e;
    if ((e = dalloc(h, &h->merge.changed, h->cap)) != cudaSuccess) return e;
    if ((e = dalloc(h, &h->merge.a, p2)) != cudaSuccess) return e;
    if ((e = dalloc(h, &h->merge.b, p2)) != cudaSuccess) return e;
    if ((e = dalloc(h, &h->merge.count, 2)) != cudaSuccess) return e;
    if ((e = merge_sort_setup()) != cudaSuccess) return e;
    h->merge_ready = true;
    return cudaSuccess;
}

// cell rows on each side along y and z that cover one cell_size
static int walk_reach(float cell_size, float cell_yz) {
    return cell_yz < cell_size ? (int)std::ceil((double)cell_size / (double)cell_yz - 1e-9) : 1;
}

// the fluid list's capacity: every fluid particle, and one gap for each warp
// of a gather over cap particles (blocks of 256) that can hold fluid
static uint32_t fluid_list_cap(uint32_t nfluid, uint32_t cap) {
    const uint64_t warps = ((uint64_t)cap + 255) / 256 * 8;
    const uint64_t gaps = warps < nfluid ? warps : nfluid;
    const uint64_t c = (uint64_t)nfluid + gaps;
    return c > 0 ? (uint32_t)c : 1u;
}

static Grid device_grid(const HostGrid& hg, uint32_t base) {
    Grid g;
    g.left = hg.left;
    g.back = hg.back;
    g.bottom = hg.bottom;
    g.cell_size = hg.cell_size;
    g.cdx = hg.cdx;
    g.cdy = hg.cdy;
    g.cdz = hg.cdz;
    g.sheet = hg.sheet;
    g.ncells = hg.ncells;
    g.dim = hg.dim;
    g.base = base;
    g.cell_yz = hg.cell_yz;
    g.reach = walk_reach(hg.cell_size, hg.cell_yz);
    return g;
}

// cells along x and along y/z that cover sqrt(2) r0 (the dummy-to-wall search)
static void normal_reaches(double rzero, const HostGrid& hg, int* rx, int* ryz) {
    const double need = std::sqrt(2.0) * rzero;
    const int a = (int)std::ceil(need / (double)hg.cell_size - 1e-12);
    const int b = (int)std::ceil(need / (double)hg.cell_yz - 1e-12);
    *rx = a > *rx ? a : *rx;
    *ryz = b > *ryz ? b : *ryz;
}

static mps_status setup(mps_handle* h, const mps_params& prm, uint32_t np, uint32_t nb2, uint32_t nb1,
                        const float* pos3, const float* vel3, const float* press) {
    h->prm = prm;
    h->np0 = np;
    h->nb2 = nb2;
    h->nb1 = nb1;
    h->cap = h->opt.capacity > np ? h->opt.capacity : np;
    CK(cudaSetDevice(h->opt.device));
    h->dev = h->opt.device;
    CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    CK(cudaEventCreate(&h->ev0));
    CK(cudaEventCreate(&h->ev1));
    int st = make_grid(prm, pos3, np, &h->hg, &h->err);
    if (st != MPS_OK) return (mps_status)st;
    if (h->opt.arith == MPS_ARITH_FAST) refine_grid_yz(&h->hg);
    h->g = device_grid(h->hg, 0);
    const Grid& g = h->g;
    h->passes = sort_passes(g.ncells);
    h->normal_reach = h->normal_reach_yz = 1;
    normal_reaches(prm.rzero, h->hg, &h->normal_reach, &h->normal_reach_yz);

    const uint32_t cap = h->cap;
    for (int b = 0; b < 2; b++) {
        State& s = h->S[b];
        CK(dalloc(h, &s.pos, cap));
        CK(dalloc(h, &s.vel, cap));
        CK(dalloc(h, &s.press, cap));
        CK(dalloc(h, &s.n, cap));
        CK(dalloc(h, &s.id, cap));
        CK(dalloc(h, &s.cell, cap));
    }
    CK(dalloc(h, &h->tmp, cap));
    CK(dalloc(h, &h->index_of_id, cap));
    CK(dalloc(h, &h->normal_id_of, cap));
    // fluid and wall particles never change type (only drop out), so the
    // lists never outgrow the initial counts
    h->cap_fluid = np - nb2 - nb1;
    h->cap_solid = np - nb2;
    h->cap_flist = fluid_list_cap(h->cap_fluid, cap);
    CK(dalloc(h, &h->list_fluid, h->cap_flist));
    CK(dalloc(h, &h->list_solid, h->cap_solid > 0 ? h->cap_solid : 1));
    for (int b = 0; b < 2; b++) CK(dalloc(h, &h->cell_tab[b], (size_t)g.ncells + 1));
    CK(merge_setup(h));
    h->sort.tiles = sort_tiles(cap);
    for (int b = 0; b < 2; b++) {
        CK(dalloc(h, &h->sort.keys[b], cap));
        CK(dalloc(h, &h->sort.vals[b], cap));
    }
    CK(dalloc(h, &h->sort.hist, (size_t)SORT_RADIX * h->sort.tiles));
    CK(dalloc(h, &h->stage.pos3, 3 * (size_t)cap));
    CK(dalloc(h, &h->stage.vel3, 3 * (size_t)cap));
    CK(dalloc(h, &h->stage.press, cap));
    CK(dalloc(h, &h->stage.n, cap));
    CK(dalloc(h, &h->stage.id, cap));
    CK(dalloc(h, &h->stage.type, cap));
    CK(dalloc(h, &h->sc, 1));
    CK(dalloc(h, &h->best, 1));
    CK(dalloc(h, &h->lambda_dev, 1));

    // upload in GEO.dat order: type from the b2 / b1 / fluid ranges
    {
        std::vector<float4> p4(np), v4(np);
        std::vector<uint32_t> ids(np);
        for (uint32_t i = 0; i < np; i++) {
            const uint32_t t = i < nb2 ? T_DUMMY : (i < nb2 + nb1 ? T_WALL : T_FLUID);
            float w;
            memcpy(&w, &t, 4);
            p4[i] = make_float4(pos3[3 * i], pos3[3 * i + 1], pos3[3 * i + 2], w);
            v4[i] = make_float4(vel3 ? vel3[3 * i] : 0.f, vel3 ? vel3[3 * i + 1] : 0.f, vel3 ? vel3[3 * i + 2] : 0.f, 0.f);
            ids[i] = i;
        }
        State& s = h->S[0];
        CK(cudaMemcpyAsync(s.pos, p4.data(), np * sizeof(float4), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(s.vel, v4.data(), np * sizeof(float4), cudaMemcpyHostToDevice, h->stream));
        if (press) CK(cudaMemcpyAsync(s.press, press, np * sizeof(float), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(s.id, ids.data(), np * sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream));
        Scalars sc0;
        memset(&sc0, 0, sizeof sc0);
        sc0.np = np;
        sc0.np_new = np;
        sc0.dt = prm.dt_max;
        sc0.g_eff[2] = -9.81f;
        CK(cudaMemcpyAsync(h->sc, &sc0, sizeof sc0, cudaMemcpyHostToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }

    // constants that do not depend on n0
    Phys& P = h->P;
    P = base_phys(prm);

    // MPS_GPU::Initial (MPS_CAL_expl_v1.0/MPS_GPU.cpp:63-115): divideCell, then calOnce.
    rebuild(h, APPLY_NONE);
    if (h->opt.method == MPS_METHOD_SEMI_IMPLICIT) {
        // MPS_CPU::Initial / MPS::calOnce of MPS_CAL_v4.0 (MPS_CPU.cpp:54-122,
        // MPS.cpp:305-370): n of every particle, n0, lambda, in double
        double* n64 = nullptr;
        double* res = nullptr;
        CK(dalloc(h, &n64, cap));
        CK(dalloc(h, &res, 2));
        StageArgs a = stage_args(h);
        launch_pnd64(a, n64, h->cap, h->stream);
        launch_n0_lambda64(a, n64, res, h->stream);
        launch_normals(a, h->normal_reach, h->normal_reach_yz, h->normal_id_of, h->cap, h->stream);
        double hr[2] = {0, 0};
        CK(cudaMemcpyAsync(hr, res, sizeof hr, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        CK(cudaGetLastError());
        if (!(hr[0] > 0.0)) {
            h->err = "n0 is not positive: no particle has a neighbour within r0";
            return MPS_ERR_INVALID;
        }
        h->ppe.n0_64 = hr[0];
        h->ppe.lambda64 = hr[1];
        h->hc = semi_constants(prm, hr[0], hr[1]);
    } else {
        StageArgs a = stage_args(h);
        launch_pnd(a, 0, 1, h->cap, h->stream);  // n of every particle
        launch_nzero(h->S[h->cur].n, h->sc, h->best, h->cap, h->stream);
        launch_lambda(a, h->best, h->lambda_dev, h->stream);
        launch_normals(a, h->normal_reach, h->normal_reach_yz, h->normal_id_of, h->cap, h->stream);
        unsigned long long best = 0;
        float lam = 0.f;
        CK(cudaMemcpyAsync(&best, h->best, 8, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaMemcpyAsync(&lam, h->lambda_dev, 4, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        CK(cudaGetLastError());
        uint32_t nbits = (uint32_t)(best >> 32);
        float n0;
        memcpy(&n0, &nbits, 4);
        if (!(n0 > 0.f)) {
            h->err = "n0 is not positive: no particle has a neighbour within r0";
            return MPS_ERR_INVALID;
        }
        derive_constants(prm, n0, lam, &h->hc);
    }
    apply_constants(P, h->hc);

    if (h->opt.rebuild_merge != 0 && h->opt.rebuild_merge != -1) {
        h->err = "rebuild_merge is 0 (merge when few particles can move) or -1 (always sort)";
        return MPS_ERR_INVALID;
    }
    if (h->opt.visc_implicit && h->opt.method != MPS_METHOD_SEMI_IMPLICIT) {
        h->err = "Crank-Nicolson viscosity needs the semi-implicit method";
        return MPS_ERR_INVALID;
    }
    if (h->opt.method == MPS_METHOD_SEMI_IMPLICIT) {
        int e = ppe_setup(h->ppe, h->cap, h->g, h->P, h->prm, h->stream, &h->err);
        if (e != MPS_OK) return (mps_status)e;
        h->ppe.pipelined = h->opt.ppe_pipelined != 0;
        size_t keep_bytes = (size_t)h->opt.ppe_l2_keep_mb << 20;
        if (h->opt.ppe_l2_keep_mb == 0) {  // half the L2: the best of a sweep at 310,912 particles
            int l2 = 0;
            cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, h->opt.device);
            keep_bytes = (size_t)l2 / 2;
        }
        h->ppe.l2_keep_entries = h->opt.ppe_l2_keep_mb < 0 ? 0xFFFFFFFFu : (uint32_t)(keep_bytes / 8);
        if (h->opt.precond == MPS_PRECOND_LEARNED) {
            e = ppe_enable_learned(h->ppe, &h->err);
            if (e == MPS_OK) e = ppe_sp_enable(h->ppe, &h->err);
            if (e != MPS_OK) return (mps_status)e;
        }
        if (h->opt.ppe_layout != 0 && h->opt.ppe_layout != -1) {
            h->err = "ppe_layout is 0 (compact where it applies) or -1 (8-byte layout)";
            return MPS_ERR_INVALID;
        }
        h->ppe.c16_smem_chunks = h->opt.ppe_smem_chunks == 0 ? 8 : (h->opt.ppe_smem_chunks < 0 ? 0 : h->opt.ppe_smem_chunks);
        h->ppe.precond_every = h->opt.precond_every > 0 ? h->opt.precond_every : 40;
        h->ppe.index_of_id = h->index_of_id;
        if (h->opt.ppe_layout == 0 && !h->nscenes) {
            e = ppe_c16_enable(h->ppe, &h->err);
            if (e != MPS_OK) return (mps_status)e;
            if (h->opt.precond == MPS_PRECOND_LEARNED) {
                e = ppe_c16_learned_enable(h->ppe, &h->err);
                if (e != MPS_OK) return (mps_status)e;
            }
            set_compact(h, true);
        }
        if (h->opt.visc_implicit) {
            e = ppe_setup(h->cn, h->cap, h->g, h->P, h->prm, h->stream, &h->err);
            if (e != MPS_OK) return (mps_status)e;
            h->cn.write_pressure = false;
            h->cn.l2_keep_entries = h->ppe.l2_keep_entries;
        }
    }
    Scalars s;
    return read_status(h, &s);
}

static mps_status create_common(mps_handle** out, const mps_options* opt) {
    mps_handle* h = new mps_handle();
    if (opt) h->opt = *opt;
    else mps_default_options(&h->opt);
    if (h->opt.cg_max_iter <= 0) h->opt.cg_max_iter = 10000;
    if (h->opt.cg_check_every <= 0) h->opt.cg_check_every = 1000;
    if (h->opt.cg_inner_digits <= 0) h->opt.cg_inner_digits = 4;
    if (h->opt.cg_tol <= 0) h->opt.cg_tol = 1e-8;
    *out = h;
    return MPS_OK;
}

extern "C" mps_status mps_create(const char* input_dat, const char* geo_dat, const mps_options* opt,
                                 mps_handle** out) {
    if (!out || !input_dat || !geo_dat) return MPS_ERR_INVALID;
    *out = nullptr;
    mps_handle* h;
    create_common(&h, opt);
    mps_params p;
    int st = read_input_dat(input_dat, &p, &h->err);
    Geo geo;
    if (st == MPS_OK) st = read_geo_dat(geo_dat, &geo, &h->err);
    if (st == MPS_OK)
        st = setup(h, p, geo.np, geo.nb2, geo.nb1, geo.pos.data(), geo.vel.data(), geo.press.data());
    *out = h;  // returned even on error so that mps_last_error can explain
    return (mps_status)st;
}

extern "C" mps_status mps_create_from_arrays(const mps_params* p, uint32_t np, uint32_t nb2, uint32_t nb1,
                                             const float* pos3, const float* vel3, const float* press,
                                             const mps_options* opt, mps_handle** out) {
    if (!out || !p || !pos3 || np == 0 || nb2 + nb1 > np) return MPS_ERR_INVALID;
    mps_handle* h;
    create_common(&h, opt);
    int st = setup(h, *p, np, nb2, nb1, pos3, vel3, press);
    *out = h;
    return (mps_status)st;
}

// ---------------------------------------------------------------- batch
// A batch is one particle set made of the scenes' particles (ids offset by
// the earlier scenes' counts), one cell space made of each scene's own grid
// (offset by the earlier grids' cells), and per-scene constants and step
// scalars.  Every stage kernel runs once over all scenes; a particle reads
// its scene's grid, constants and dt, so each scene evolves as it would
// alone.
static mps_status setup_batch(mps_handle* h, const std::vector<mps_params>& prms, const std::vector<Geo>& geos,
                              const mps_scene_spec* specs) {
    const uint32_t S = (uint32_t)prms.size();
    for (uint32_t s = 1; s < S; s++)
        if (prms[s].dim != prms[0].dim) {
            h->err = "every scene of a batch must have the same dimension";
            return MPS_ERR_INVALID;
        }
    h->prm = prms[0];
    h->nscenes = S;
    uint64_t np64 = 0;
    h->id_base.assign(S + 1, 0);
    h->nb2 = h->nb1 = 0;
    uint32_t nfluid = 0;
    for (uint32_t s = 0; s < S; s++) {
        h->id_base[s] = (uint32_t)np64;
        np64 += geos[s].np;
        h->nb2 += geos[s].nb2;
        h->nb1 += geos[s].nb1;
        nfluid += geos[s].np - geos[s].nb2 - geos[s].nb1;
        h->scene_nb2.push_back(geos[s].nb2);
        h->scene_nb1.push_back(geos[s].nb1);
    }
    if (np64 >= 0xffffffffull) {
        h->err = "too many particles in the batch";
        return MPS_ERR_INVALID;
    }
    const uint32_t np = (uint32_t)np64;
    h->id_base[S] = np;
    h->np0 = np;
    h->cap = h->opt.capacity > np ? h->opt.capacity : np;
    CK(cudaSetDevice(h->opt.device));
    h->dev = h->opt.device;
    CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    CK(cudaEventCreate(&h->ev0));
    CK(cudaEventCreate(&h->ev1));
    // per-scene grids in one cell space
    uint64_t cells = 0;
    int reach = 1, reach_yz = 1;
    for (uint32_t s = 0; s < S; s++) {
        HostGrid hg;
        int st = make_grid(prms[s], geos[s].pos.data(), geos[s].np, &hg, &h->err);
        if (st != MPS_OK) {
            h->err = "scene " + std::to_string(s) + ": " + h->err;
            return (mps_status)st;
        }
        if (h->opt.arith == MPS_ARITH_FAST) refine_grid_yz(&hg);
        if (s == 0) h->hg = hg;
        h->scene_grid.push_back(device_grid(hg, (uint32_t)cells));
        cells += hg.ncells;
        normal_reaches(prms[s].rzero, hg, &reach, &reach_yz);
    }
    if (cells >= 0xffffffffull) {
        h->err = "too many cells in the batch";
        return MPS_ERR_INVALID;
    }
    h->g = h->scene_grid[0];
    h->g.ncells = (uint32_t)cells;  // the whole cell space (cell table and sort)
    h->g.base = 0;
    h->passes = sort_passes(h->g.ncells);
    h->normal_reach = reach;
    h->normal_reach_yz = reach_yz;

    const uint32_t cap = h->cap;
    for (int b = 0; b < 2; b++) {
        State& st = h->S[b];
        CK(dalloc(h, &st.pos, cap));
        CK(dalloc(h, &st.vel, cap));
        CK(dalloc(h, &st.press, cap));
        CK(dalloc(h, &st.n, cap));
        CK(dalloc(h, &st.id, cap));
        CK(dalloc(h, &st.cell, cap));
    }
    CK(dalloc(h, &h->tmp, cap));
    CK(dalloc(h, &h->index_of_id, cap));
    CK(dalloc(h, &h->normal_id_of, cap));
    h->cap_fluid = nfluid;
    h->cap_solid = np - h->nb2;
    h->cap_flist = fluid_list_cap(h->cap_fluid, cap);
    CK(dalloc(h, &h->list_fluid, h->cap_flist));
    CK(dalloc(h, &h->list_solid, h->cap_solid > 0 ? h->cap_solid : 1));
    for (int b = 0; b < 2; b++) CK(dalloc(h, &h->cell_tab[b], (size_t)h->g.ncells + 1));
    CK(merge_setup(h));
    h->sort.tiles = sort_tiles(cap);
    for (int b = 0; b < 2; b++) {
        CK(dalloc(h, &h->sort.keys[b], cap));
        CK(dalloc(h, &h->sort.vals[b], cap));
    }
    CK(dalloc(h, &h->sort.hist, (size_t)SORT_RADIX * h->sort.tiles));
    CK(dalloc(h, &h->stage.pos3, 3 * (size_t)cap));
    CK(dalloc(h, &h->stage.vel3, 3 * (size_t)cap));
    CK(dalloc(h, &h->stage.press, cap));
    CK(dalloc(h, &h->stage.n, cap));
    CK(dalloc(h, &h->stage.id, cap));
    CK(dalloc(h, &h->stage.type, cap));
    CK(dalloc(h, &h->sc, 1));
    CK(dalloc(h, &h->best, 1));
    CK(dalloc(h, &h->lambda_dev, 1));
    // scene tables
    uint32_t* sid = nullptr;
    Grid* grid_dev = nullptr;
    CK(dalloc(h, &sid, np));
    CK(dalloc(h, &grid_dev, S));
    CK(dalloc(h, &h->phys_dev, S));
    CK(dalloc(h, &h->batch.dt, S));
    CK(dalloc(h, &h->batch.time, S));
    CK(dalloc(h, &h->batch.g_eff, S));
    CK(dalloc(h, &h->batch.vmax2_bits, S));
    h->batch.n = S;
    h->batch.sid_of_id = sid;
    h->batch.grid = grid_dev;
    h->batch.phys = h->phys_dev;
    h->batch.ncells = h->g.ncells;
    for (uint32_t s = 0; s < S; s++) {
        Phys P = base_phys(prms[s]);
        P.body_amp = (double)specs[s].accel_amp;
        P.body_omega = 2.0 * M_PI * (double)specs[s].accel_freq;
        h->scene_phys.push_back(P);
    }
    {
        std::vector<float4> p4(np), v4(np);
        std::vector<uint32_t> ids(np), sids(np);
        std::vector<float> pr(np, 0.f), dts(S), times(S, 0.f);
        std::vector<float4> ge(S, make_float4(0.f, 0.f, -9.81f, 0.f));
        for (uint32_t s = 0; s < S; s++) {
            const Geo& g = geos[s];
            for (uint32_t k = 0; k < g.np; k++) {
                const uint32_t i = h->id_base[s] + k;
                const uint32_t t = k < g.nb2 ? T_DUMMY : (k < g.nb2 + g.nb1 ? T_WALL : T_FLUID);
                float w;
                memcpy(&w, &t, 4);
                p4[i] = make_float4(g.pos[3 * k], g.pos[3 * k + 1], g.pos[3 * k + 2], w);
                v4[i] = make_float4(g.vel[3 * k], g.vel[3 * k + 1], g.vel[3 * k + 2], 0.f);
                pr[i] = g.press[k];
                ids[i] = i;
                sids[i] = s;
            }
            dts[s] = prms[s].dt_max;
        }
        State& st0 = h->S[0];
        CK(cudaMemcpyAsync(st0.pos, p4.data(), np * sizeof(float4), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(st0.vel, v4.data(), np * sizeof(float4), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(st0.press, pr.data(), np * sizeof(float), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(st0.id, ids.data(), np * sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(sid, sids.data(), np * sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(grid_dev, h->scene_grid.data(), S * sizeof(Grid), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(h->phys_dev, h->scene_phys.data(), S * sizeof(Phys), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(h->batch.dt, dts.data(), S * sizeof(float), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(h->batch.time, times.data(), S * sizeof(float), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(h->batch.g_eff, ge.data(), S * sizeof(float4), cudaMemcpyHostToDevice, h->stream));
        Scalars sc0;
        memset(&sc0, 0, sizeof sc0);
        sc0.np = np;
        sc0.np_new = np;
        sc0.dt = prms[0].dt_max;
        sc0.g_eff[2] = -9.81f;
        CK(cudaMemcpyAsync(h->sc, &sc0, sizeof sc0, cudaMemcpyHostToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    h->P = h->scene_phys[0];

    // initial rebuild, then each scene's n0 and lambda from its own particles
    rebuild(h, APPLY_NONE);
    std::vector<uint32_t> lo(S), hi(S);
    for (uint32_t s = 0; s < S; s++) {
        const Grid& g = h->scene_grid[s];
        CK(cudaMemcpyAsync(&lo[s], h->cell_tab[h->cur] + g.base, 4, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaMemcpyAsync(&hi[s], h->cell_tab[h->cur] + g.base + g.ncells, 4, cudaMemcpyDeviceToHost, h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
    std::vector<PpeScene> ppe_scenes(S);
    StageArgs a = stage_args(h);
    if (h->opt.method == MPS_METHOD_SEMI_IMPLICIT) {
        double* n64 = nullptr;
        double* res = nullptr;
        CK(dalloc(h, &n64, cap));
        CK(dalloc(h, &res, 2 * (size_t)S));
        launch_pnd64(a, n64, cap, h->stream);
        for (uint32_t s = 0; s < S; s++) launch_n0_lambda64(a, n64, res + 2 * s, h->stream, lo[s], hi[s]);
        std::vector<double> hr(2 * (size_t)S);
        CK(cudaMemcpyAsync(hr.data(), res, hr.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        CK(cudaGetLastError());
        for (uint32_t s = 0; s < S; s++) {
            const double n0 = hr[2 * s], lam = hr[2 * s + 1];
            if (!(n0 > 0.0)) {
                h->err = "scene " + std::to_string(s) + ": n0 is not positive";
                return MPS_ERR_INVALID;
            }
            const mps_params& q = prms[s];
            const HostConst c = semi_constants(q, n0, lam);
            h->scene_hc.push_back(c);
            apply_constants(h->scene_phys[s], c);
            const double rho = (double)q.rho, dim = (double)q.dim;
            const double alpha = 1.0 / (rho * (double)q.cs * (double)q.cs);
            const double one_over_dt = 1.0 / (double)q.dt_max;
            ppe_scenes[s].n0 = n0;
            ppe_scenes[s].beta = (double)q.beta;
            ppe_scenes[s].b_tmp = lam * rho * (0.5 * (1.0 / dim) * one_over_dt * one_over_dt);
            ppe_scenes[s].rho_lambda_alpha_n0 = rho * lam * alpha * n0;
        }
        h->ppe.n0_64 = ppe_scenes[0].n0;
        h->ppe.lambda64 = hr[1];
    } else {
        launch_pnd(a, 0, 1, cap, h->stream);
        for (uint32_t s = 0; s < S; s++) {
            CK(cudaMemsetAsync(h->best, 0, sizeof(unsigned long long), h->stream));
            launch_nzero_range(h->S[h->cur].n, lo[s], hi[s], h->best, h->stream);
            launch_lambda(a, h->best, h->lambda_dev, h->stream);
            unsigned long long best = 0;
            float lam = 0.f;
            CK(cudaMemcpyAsync(&best, h->best, 8, cudaMemcpyDeviceToHost, h->stream));
            CK(cudaMemcpyAsync(&lam, h->lambda_dev, 4, cudaMemcpyDeviceToHost, h->stream));
            CK(cudaStreamSynchronize(h->stream));
            CK(cudaGetLastError());
            const uint32_t nbits = (uint32_t)(best >> 32);
            float n0;
            memcpy(&n0, &nbits, 4);
            if (!(n0 > 0.f)) {
                h->err = "scene " + std::to_string(s) + ": n0 is not positive";
                return MPS_ERR_INVALID;
            }
            HostConst c;
            derive_constants(prms[s], n0, lam, &c);
            h->scene_hc.push_back(c);
            apply_constants(h->scene_phys[s], c);
        }
    }
    launch_normals(a, h->normal_reach, h->normal_reach_yz, h->normal_id_of, cap, h->stream);
    CK(cudaMemcpyAsync(h->phys_dev, h->scene_phys.data(), S * sizeof(Phys), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->P = h->scene_phys[0];
    h->hc = h->scene_hc[0];
    if (h->opt.method == MPS_METHOD_SEMI_IMPLICIT) {
        int e = ppe_setup(h->ppe, cap, h->g, h->P, h->prm, h->stream, &h->err);
        if (e != MPS_OK) return (mps_status)e;
        e = ppe_setup_batch(h->ppe, ppe_scenes.data(), S, h->stream, &h->err);
        if (e != MPS_OK) return (mps_status)e;
        h->ppe.precond_every = h->opt.precond_every > 0 ? h->opt.precond_every : 40;
        h->ppe.index_of_id = h->index_of_id;
        if (h->opt.precond == MPS_PRECOND_LEARNED) {
            e = ppe_enable_learned(h->ppe, &h->err);
            if (e == MPS_OK) e = ppe_sp_enable(h->ppe, &h->err);
            if (e != MPS_OK) return (mps_status)e;
        }
    }
    Scalars sc;
    return read_status(h, &sc);
}

extern "C" mps_status mps_batch_create(const mps_scene_spec* scenes, uint32_t nscenes, const mps_options* opt,
                                       mps_handle** out) {
    if (!out || !scenes || nscenes == 0) return MPS_ERR_INVALID;
    *out = nullptr;
    mps_handle* h;
    create_common(&h, opt);
    *out = h;
    if (nscenes > PPE_MAX_SCENES) {
        h->err = "a batch holds at most " + std::to_string(PPE_MAX_SCENES) + " scenes";
        return MPS_ERR_INVALID;
    }
    if (h->opt.visc_implicit) {
        h->err = "Crank-Nicolson viscosity is for single-scene handles";
        return MPS_ERR_INVALID;
    }
    std::vector<mps_params> prms(nscenes);
    std::vector<Geo> geos(nscenes);
    for (uint32_t s = 0; s < nscenes; s++) {
        if (!scenes[s].input_dat || !scenes[s].geo_dat) return MPS_ERR_INVALID;
        int st = read_input_dat(scenes[s].input_dat, &prms[s], &h->err);
        if (st == MPS_OK) st = read_geo_dat(scenes[s].geo_dat, &geos[s], &h->err);
        if (st != MPS_OK) {
            h->err = "scene " + std::to_string(s) + ": " + h->err;
            return (mps_status)st;
        }
    }
    return setup_batch(h, prms, geos, scenes);
}

extern "C" mps_status mps_batch_step(mps_handle* h, int nsteps, mps_step_stats* stats) {
    return mps_step(h, nsteps, stats);
}

extern "C" mps_status mps_batch_scene_info(mps_handle* h, uint32_t scene, mps_scene_info* info) {
    if (!h || !info) return MPS_ERR_INVALID;
    const uint32_t S = h->nscenes ? h->nscenes : 1;
    if (scene >= S) return MPS_ERR_INVALID;
    CK(cudaSetDevice(h->dev));
    Scalars sc;
    mps_status st = read_status(h, &sc);
    if (st == MPS_ERR_CUDA) return st;
    memset(info, 0, sizeof *info);
    if (!h->nscenes) {
        info->id_base = 0;
        info->np0 = h->np0;
        info->nb2 = h->nb2;
        info->nb1 = h->nb1;
        info->time = sc.time;
        info->dt = sc.dt;
        info->cg_iters = sc.cg_iters;
        info->cg_outer = sc.cg_outer;
        info->cg_relres = sc.cg_relres;
        info->nzero = h->hc.nzero;
        return MPS_OK;
    }
    info->id_base = h->id_base[scene];
    info->np0 = h->id_base[scene + 1] - h->id_base[scene];
    info->nb2 = h->scene_nb2[scene];
    info->nb1 = h->scene_nb1[scene];
    info->nzero = h->scene_hc[scene].nzero;
    cudaStream_t s = h->stream;
    CK(cudaMemcpyAsync(&info->time, h->batch.time + scene, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&info->dt, h->batch.dt + scene, 4, cudaMemcpyDeviceToHost, s));
    if (h->opt.method == MPS_METHOD_SEMI_IMPLICIT && h->ppe.scene_iters) {
        CK(cudaMemcpyAsync(&info->cg_iters, h->ppe.scene_iters + scene, 4, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(&info->cg_outer, h->ppe.scene_outer + scene, 4, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(&info->cg_relres, h->ppe.scene_relres + scene, 8, cudaMemcpyDeviceToHost, s));
    }
    CK(cudaStreamSynchronize(s));
    return MPS_OK;
}

extern "C" mps_status mps_set_body_force(mps_handle* h, uint32_t scene, float accel_amp, float accel_freq) {
    if (!h) return MPS_ERR_INVALID;
    CK(cudaSetDevice(h->dev));
    const double amp = (double)accel_amp, omega = 2.0 * M_PI * (double)accel_freq;
    if (h->nscenes) {
        if (scene >= h->nscenes) return MPS_ERR_INVALID;
        h->scene_phys[scene].body_amp = amp;
        h->scene_phys[scene].body_omega = omega;
        CK(cudaMemcpyAsync(h->phys_dev + scene, &h->scene_phys[scene], sizeof(Phys), cudaMemcpyHostToDevice,
                           h->stream));
        CK(cudaStreamSynchronize(h->stream));
        return MPS_OK;
    }
    if (scene != 0) return MPS_ERR_INVALID;
    h->P.body_amp = amp;
    h->P.body_omega = omega;
    // the captured steps hold the old constants
    CK(cudaStreamSynchronize(h->stream));
    drop_graphs(h);
    return MPS_OK;
}

extern "C" mps_status mps_set_device_wait_limit(mps_handle* h, uint64_t ns) {
    if (!h) return MPS_ERR_INVALID;
    CK(cudaSetDevice(h->dev));
    const unsigned long long v = ns;
    CK(cudaMemcpyAsync(reinterpret_cast<char*>(h->sc) + offsetof(Scalars, wait_ns), &v, sizeof v,
                       cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return MPS_OK;
}

// ---------------------------------------------------------------- boundary motion
extern "C" mps_status mps_add_wall_motion(mps_handle* h, const float lo[3], const float hi[3], const float vel[3],
                                          const float amp[3], float freq, float phase, uint32_t* selected) {
    if (!h || !lo || !hi || !vel || !amp) return MPS_ERR_INVALID;
    if (h->nscenes) {
        h->err = "wall motions are for single-scene handles";
        return MPS_ERR_INVALID;
    }
    if (h->mot.n >= MPS_MAX_MOTIONS) {
        h->err = "at most " + std::to_string(MPS_MAX_MOTIONS) + " wall motions";
        return MPS_ERR_INVALID;
    }
    CK(cudaSetDevice(h->dev));
    if (!h->motion_of) {
        CK(dalloc(h, &h->motion_of, h->cap));
        CK(dalloc(h, &h->motion_x0, h->cap));
        CK(dalloc(h, &h->motion_count, 1));
        CK(cudaMemsetAsync(h->motion_of, 0xFF, (size_t)h->cap * 4, h->stream));
    }
    const int m = h->mot.n;
    CK(cudaMemsetAsync(h->motion_count, 0, 4, h->stream));
    launch_motion_select(h->S[h->cur], h->sc, lo, hi, (uint32_t)m, h->motion_of, h->motion_x0, h->motion_count,
                         h->cap, h->stream);
    CK(cudaGetLastError());
    uint32_t count = 0;
    Scalars sc;
    CK(cudaMemcpyAsync(&count, h->motion_count, 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(&sc, h->sc, sizeof sc, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->mot.t0[m] = (double)sc.time;
    for (int c = 0; c < 3; c++) {
        h->mot.vel[m][c] = (double)vel[c];
        h->mot.amp[m][c] = (double)amp[c];
    }
    h->mot.omega[m] = 2.0 * M_PI * (double)freq;
    h->mot.phase[m] = (double)phase;
    h->mot.n = m + 1;
    h->moving += count;
    if (selected) *selected = count;
    drop_graphs(h);  // the captured steps hold the old motion set
    return MPS_OK;
}

extern "C" mps_status mps_clear_wall_motion(mps_handle* h) {
    if (!h) return MPS_ERR_INVALID;
    CK(cudaSetDevice(h->dev));
    if (h->motion_of) {
        launch_motion_stop(h->S[h->cur], h->sc, h->motion_of, h->cap, h->stream);
        CK(cudaGetLastError());
        CK(cudaMemsetAsync(h->motion_of, 0xFF, (size_t)h->cap * 4, h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
    h->mot.n = 0;
    h->moving = 0;
    drop_graphs(h);
    return MPS_OK;
}

extern "C" void mps_destroy(mps_handle* h) {
    if (!h) return;
    cudaSetDevice(h->dev);
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (int b = 0; b < 2; b++)
        if (h->graph[b]) cudaGraphExecDestroy(h->graph[b]);
    for (int b = 2; b < 4; b++)
        if (h->graph[b]) cudaGraphExecDestroy(h->graph[b]);
    for (cudaEvent_t e : h->prof_ev) cudaEventDestroy(e);
    ppe_free(h->ppe);
    ppe_free(h->cn);
    surface_free(h->surf);
    for (void* p : h->allocs) cudaFree(p);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

extern "C" const char* mps_last_error(mps_handle* h) { return h ? h->err.c_str() : "null handle"; }

// ---------------------------------------------------------------- stepping
// Before every step: whether it evaluates the learned network (the learned
// preconditioner re-evaluates it every precond_every steps); false for every
// other configuration.
static bool begin_step(mps_handle* h) {
    if (h->opt.method != MPS_METHOD_SEMI_IMPLICIT || h->opt.precond != MPS_PRECOND_LEARNED || !h->ppe.lp.ready ||
        !h->ppe.sp_ent)
        return false;
    return ppe_begin_step(h->ppe);
}

static mps_status capture_graph(mps_handle* h, int parity, int slot) {
    cudaGraph_t g;
    const int saved = h->cur;
    h->cur = parity;
    CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    enqueue_step(h);
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    const int after = h->cur;
    h->cur = saved;
    if (e != cudaSuccess) {
        h->err = std::string("graph capture: ") + cudaGetErrorString(e);
        return MPS_ERR_CUDA;
    }
    if (after != (parity ^ 1)) {
        cudaGraphDestroy(g);
        h->err = "unexpected buffer parity after a step";
        return MPS_ERR_INVALID;
    }
    e = cudaGraphInstantiate(&h->graph[slot], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        h->err = std::string("graph instantiate: ") + cudaGetErrorString(e);
        return MPS_ERR_CUDA;
    }
    return MPS_OK;
}

static void drop_graphs(mps_handle* h) {
    for (int b = 0; b < 4; b++)
        if (h->graph[b]) {
            cudaGraphExecDestroy(h->graph[b]);
            h->graph[b] = nullptr;
        }
}

static mps_status step_async(mps_handle* h, int nsteps) {
    h->sc_valid = false;
    CK(cudaSetDevice(h->dev));
    for (int k = 0; k < nsteps; k++) {
        const bool net = begin_step(h);
        if (h->opt.use_graph && !h->graph_off) {
            const int p = h->cur;
            const int slot = p + (net ? 2 : 0);
            if (!h->graph[slot]) {
                mps_status s = capture_graph(h, p, slot);
                if (s != MPS_OK) {
                    // a capture the driver refuses falls back to direct
                    // launches; the reason stays readable
                    cudaGetLastError();
                    h->graph_off = true;
                    h->graph_note = h->err;
                    enqueue_step(h);
                    continue;
                }
            }
            CK(cudaGraphLaunch(h->graph[slot], h->stream));
            h->cur ^= 1;
        } else {
            enqueue_step(h);
        }
    }
    CK(cudaGetLastError());
    if (h->launch_err != cudaSuccess) {
        const cudaError_t e = h->launch_err;
        h->launch_err = cudaSuccess;
        h->err = std::string("cooperative PPE launch: ") + cudaGetErrorString(e);
        return MPS_ERR_CUDA;
    }
    return MPS_OK;
}

extern "C" mps_status mps_step(mps_handle* h, int nsteps, mps_step_stats* stats) {
    if (!h || nsteps < 0) return MPS_ERR_INVALID;
    if (h->pending_apply != APPLY_NONE) {
        h->err = "a stage update is pending; run stage 2 (divideCell) first";
        return MPS_ERR_INVALID;
    }
    CK(cudaEventRecord(h->ev0, h->stream));
    mps_status s = step_async(h, nsteps);
    if (s != MPS_OK) return s;
    CK(cudaEventRecord(h->ev1, h->stream));
    Scalars sc;
    s = read_status(h, &sc);
    if (stats) {
        memset(stats, 0, sizeof *stats);
        stats->np = sc.np;
        stats->nexcl = sc.nexcl;
        stats->step = sc.step;
        stats->time = sc.time;
        stats->dt = sc.dt;
        stats->cg_iters = sc.cg_iters;
        stats->cg_relres = sc.cg_relres;
        stats->cg_outer = (uint32_t)sc.cg_outer;
        stats->status = (int)s;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, h->ev0, h->ev1);
        stats->ms = ms;
    }
    return s;
}

extern "C" mps_status mps_step_async(mps_handle* h, int nsteps) {
    if (!h || nsteps < 0) return MPS_ERR_INVALID;
    if (h->pending_apply != APPLY_NONE) {
        h->err = "a stage update is pending; run stage 2 (divideCell) first";
        return MPS_ERR_INVALID;
    }
    return step_async(h, nsteps);
}

extern "C" mps_status mps_phase(mps_handle* h, int phase) {
    if (!h) return MPS_ERR_INVALID;
    CK(cudaSetDevice(h->dev));
    cudaStream_t st = h->stream;
    const uint32_t cap = h->cap;
    switch (phase) {
        case 0: launch_update_dt(stage_args(h), cap, st); break;
        case 1: launch_visc(stage_args(h), cap, st); h->pending_apply = APPLY_SET_VEL; break;
        case 2: rebuild(h, h->pending_apply); h->pending_apply = APPLY_NONE; break;
        case 3: launch_collision(stage_args(h), cap, st); h->pending_apply = APPLY_ADD_VEL; break;
        case 4: launch_pnd(stage_args(h), 0, 0, cap, st); break;
        case 5:
            launch_pnd(stage_args(h), 1, 0, cap, st);
            launch_dummy_press(stage_args(h), h->normal_id_of, h->index_of_id, cap, st);
            break;
        case 6: launch_dash(stage_args(h), cap, st); h->pending_apply = APPLY_ADD_VEL; break;
        case 7:
            if (h->opt.method != MPS_METHOD_SEMI_IMPLICIT) return MPS_ERR_INVALID;
            begin_step(h);
            ppe_enqueue_setup(h->ppe, stage_args(h), h->opt, cap, st);
            ppe_enqueue_solve(h->ppe, stage_args(h), h->opt, cap, st);
            break;
        default: return MPS_ERR_INVALID;
    }
    CK(cudaGetLastError());
    return read_status(h, nullptr);
}

// ---------------------------------------------------------------- getters
// particle counts: those of the last status read while no step or rebuild
// has been enqueued since (saves a device round trip per state transfer)
static mps_status counts(mps_handle* h, Scalars* s) {
    if (h->sc_valid) {
        *s = h->sc_host;
        return MPS_OK;
    }
    return read_status(h, s) == MPS_ERR_CUDA ? MPS_ERR_CUDA : MPS_OK;
}

extern "C" mps_status mps_get_counts(mps_handle* h, uint32_t* np, uint32_t* nb2, uint32_t* nb1, uint32_t* nexcl) {
    if (!h) return MPS_ERR_INVALID;
    Scalars s;
    if (counts(h, &s) != MPS_OK) return MPS_ERR_CUDA;
    if (np) *np = s.np;
    if (nb2) *nb2 = h->nb2;
    if (nb1) *nb1 = h->nb1;
    if (nexcl) *nexcl = s.nexcl;
    return MPS_OK;
}

extern "C" mps_status mps_get_state(mps_handle* h, uint32_t* id, uint32_t* type, float* pos3, float* vel3,
                                    float* press, float* n, int order) {
    if (!h || (order != MPS_ORDER_SORTED && order != MPS_ORDER_BY_ID)) return MPS_ERR_INVALID;
    CK(cudaSetDevice(h->dev));
    Scalars s;
    if (counts(h, &s) != MPS_OK) return MPS_ERR_CUDA;
    const int by_id = order == MPS_ORDER_BY_ID;
    const size_t cnt = by_id ? h->np0 : s.np;
    if (cnt == 0) return MPS_OK;
    cudaStream_t st = h->stream;
    launch_unpack(h->S[h->cur], h->stage, by_id, h->np0, h->sc, h->cap, st);
    if (id) CK(cudaMemcpyAsync(id, h->stage.id, cnt * 4, cudaMemcpyDeviceToHost, st));
    if (type) CK(cudaMemcpyAsync(type, h->stage.type, cnt * 4, cudaMemcpyDeviceToHost, st));
    if (pos3) CK(cudaMemcpyAsync(pos3, h->stage.pos3, cnt * 12, cudaMemcpyDeviceToHost, st));
    if (vel3) CK(cudaMemcpyAsync(vel3, h->stage.vel3, cnt * 12, cudaMemcpyDeviceToHost, st));
    if (press) CK(cudaMemcpyAsync(press, h->stage.press, cnt * 4, cudaMemcpyDeviceToHost, st));
    if (n) CK(cudaMemcpyAsync(n, h->stage.n, cnt * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    CK(cudaGetLastError());
    return MPS_OK;
}

extern "C" mps_status mps_set_state(mps_handle* h, const float* pos3, const float* vel3, const float* press,
                                    const float* n) {
    if (!h) return MPS_ERR_INVALID;
    CK(cudaSetDevice(h->dev));
    Scalars s;
    if (counts(h, &s) != MPS_OK) return MPS_ERR_CUDA;
    const size_t np = s.np;
    if (np == 0) return MPS_OK;
    cudaStream_t st = h->stream;
    int mask = 0;
    if (pos3) { CK(cudaMemcpyAsync(h->stage.pos3, pos3, np * 12, cudaMemcpyHostToDevice, st)); mask |= 1; }
    if (vel3) { CK(cudaMemcpyAsync(h->stage.vel3, vel3, np * 12, cudaMemcpyHostToDevice, st)); mask |= 2; }
    if (press) { CK(cudaMemcpyAsync(h->stage.press, press, np * 4, cudaMemcpyHostToDevice, st)); mask |= 4; }
    if (n) { CK(cudaMemcpyAsync(h->stage.n, n, np * 4, cudaMemcpyHostToDevice, st)); mask |= 8; }
    if (mask) launch_pack(h->S[h->cur], h->stage, mask, h->sc, h->cap, st);
    CK(cudaStreamSynchronize(st));
    CK(cudaGetLastError());
    return MPS_OK;
}

extern "C" mps_status mps_get_cell_tables(mps_handle* h, uint32_t* cell_of, uint32_t* start, uint32_t* end) {
    if (!h) return MPS_ERR_INVALID;
    CK(cudaSetDevice(h->dev));
    Scalars s;
    if (counts(h, &s) != MPS_OK) return MPS_ERR_CUDA;
    const uint32_t nc = h->g.ncells;
    std::vector<uint32_t> cs(nc + 1);
    CK(cudaMemcpyAsync(cs.data(), h->cell_tab[h->cur], (nc + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                       h->stream));
    if (cell_of && s.np)
        CK(cudaMemcpyAsync(cell_of, h->S[h->cur].cell, s.np * sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (uint32_t c = 0; c < nc; c++) {
        if (start) start[c] = cs[c];
        if (end) end[c] = cs[c + 1];
    }
    return MPS_OK;
}

extern "C" mps_status mps_get_grid(mps_handle* h, mps_grid* g) {
    if (!h || !g) return MPS_ERR_INVALID;
    g->left = h->g.left;
    g->back = h->g.back;
    g->bottom = h->g.bottom;
    g->cell_size = h->g.cell_size;
    g->cdx = h->g.cdx;
    g->cdy = h->g.cdy;
    g->cdz = h->g.cdz;
    g->ncells = h->g.ncells;
    g->dim = h->g.dim;
    g->cell_yz = h->g.cell_yz;
    return MPS_OK;
}

extern "C" mps_status mps_get_scalars(mps_handle* h, double* o) {
    if (!h || !o) return MPS_ERR_INVALID;
    Scalars s;
    mps_status st = read_status(h, &s);
    if (st == MPS_ERR_CUDA) return st;
    for (int k = 0; k < 16; k++) o[k] = 0.0;
    o[0] = h->hc.nzero;
    o[1] = h->hc.lambda;
    o[2] = s.dt;
    o[3] = s.time;
    o[4] = h->hc.c_lap;
    o[5] = h->hc.one_over_alpha;
    o[6] = h->hc.alpha;
    o[7] = s.cg_iters;
    o[8] = s.cg_relres;
    o[9] = s.step;
    o[10] = (double)st;
    o[11] = h->g.ncells;
    o[12] = h->launches;
    o[13] = s.cg_outer;
    o[14] = (h->opt.use_graph && !h->graph_off) ? 1.0 : 0.0;
    o[15] = -1.0;
    if (h->opt.method == MPS_METHOD_SEMI_IMPLICIT && h->ppe.c16) {
        uint32_t esc = 0;
        CK(cudaMemcpyAsync(&esc, h->ppe.c16_esc, sizeof esc, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        o[15] = esc;
    }
    return MPS_OK;
}

// ---------------------------------------------------------------- learned preconditioner
extern "C" uint32_t mps_precond_num_params(void) { return (uint32_t)LP_NPARAM; }

// batch_ok: the call works on a batch handle (inference: parameters, the
// tensor-core switch); training and snapshots take single scenes
static mps_status need_semi(mps_handle* h, bool batch_ok = false) {
    if (!h) return MPS_ERR_INVALID;
    if (h->nscenes && !batch_ok) {
        h->err = "training the learned preconditioner takes single-scene handles";
        return MPS_ERR_INVALID;
    }
    if (h->opt.method != MPS_METHOD_SEMI_IMPLICIT) {
        h->err = "the learned preconditioner belongs to the semi-implicit method";
        return MPS_ERR_INVALID;
    }
    return MPS_OK;
}

extern "C" mps_status mps_precond_get_params(mps_handle* h, float* w, uint32_t n) {
    mps_status s = need_semi(h, true);
    if (s != MPS_OK) return s;
    if (!w || n != (uint32_t)LP_NPARAM) return MPS_ERR_INVALID;
    CK(cudaSetDevice(h->dev));
    if (!h->ppe.lp.ready) {
        lp_init_params(w, 1234);
        return MPS_OK;
    }
    CK(cudaMemcpyAsync(w, h->ppe.lp.w32, n * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return MPS_OK;
}

extern "C" mps_status mps_precond_set_params(mps_handle* h, const float* w, uint32_t n) {
    mps_status s = need_semi(h, true);
    if (s != MPS_OK) return s;
    if (!w || n != (uint32_t)LP_NPARAM) return MPS_ERR_INVALID;
    CK(cudaSetDevice(h->dev));
    const bool was_ready = h->ppe.lp.ready;
    int e = ppe_enable_learned(h->ppe, &h->err);
    if (e != MPS_OK) return (mps_status)e;
    lp_upload_params(h->ppe.lp, w, h->stream);
    h->ppe.lp.s_ready = false;  // the next step evaluates the new network
    CK(cudaStreamSynchronize(h->stream));
    if (!was_ready) drop_graphs(h);  // the step now also runs the network
    return MPS_OK;
}

static mps_status need_snapshot(mps_handle* h, bool batch_ok = false) {
    mps_status s = need_semi(h, batch_ok);
    if (s != MPS_OK) return s;
    if (!h->ppe.lp.ready || !h->ppe.have_snapshot) {
        h->err = "no PPE system with the learned stencil yet: enable the learned preconditioner "
                 "(option or mps_precond_set_params) and take a step first";
        return MPS_ERR_INVALID;
    }
    return MPS_OK;
}

extern "C" mps_status mps_precond_loss_grad(mps_handle* h, uint64_t seed, double* loss, float* grad) {
    mps_status s = need_snapshot(h);
    if (s != MPS_OK) return s;
    CK(cudaSetDevice(h->dev));
    const LpSystem L = ppe_lp_system(h->ppe, stage_args(h));
    if (lp_loss_grad(h->ppe.lp, L, h->opt.arith == MPS_ARITH_EXACT, seed, h->cap, h->stream) != 0)
        return MPS_ERR_CUDA;
    double lz[2] = {0, 0};
    uint32_t nrows = 0;
    CK(cudaMemcpyAsync(lz, h->ppe.lp.loss, 16, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(&nrows, h->ppe.nrows, 4, cudaMemcpyDeviceToHost, h->stream));
    if (grad) CK(cudaMemcpyAsync(grad, h->ppe.lp.grad, LP_NPARAM * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaGetLastError());
    if (loss) *loss = lp_loss_value(lz, nrows);
    return MPS_OK;
}

extern "C" mps_status mps_precond_train(mps_handle* h, int iters, float lr, uint64_t seed, double* loss_first,
                                        double* loss_last) {
    mps_status s = need_snapshot(h);
    if (s != MPS_OK) return s;
    if (iters < 0) return MPS_ERR_INVALID;
    CK(cudaSetDevice(h->dev));
    const LpSystem L = ppe_lp_system(h->ppe, stage_args(h));
    double first = 0.0, last = 0.0;
    for (int k = 0; k < iters; k++) {
        if (lp_loss_grad(h->ppe.lp, L, h->opt.arith == MPS_ARITH_EXACT, seed + (uint64_t)k, h->cap, h->stream) != 0)
            return MPS_ERR_CUDA;
        if (k == 0 || k == iters - 1) {
            double lz[2] = {0, 0};
            uint32_t nrows = 0;
            CK(cudaMemcpyAsync(lz, h->ppe.lp.loss, 16, cudaMemcpyDeviceToHost, h->stream));
            CK(cudaMemcpyAsync(&nrows, h->ppe.nrows, 4, cudaMemcpyDeviceToHost, h->stream));
            CK(cudaStreamSynchronize(h->stream));
            const double v = lp_loss_value(lz, nrows);
            if (k == 0) first = v;
            last = v;
        }
        lp_adam(h->ppe.lp, lr, h->stream);
    }
    // refresh G for the current system with the updated weights; the next
    // step rebuilds the preconditioner from them
    lp_forward(h->ppe.lp, L, h->opt.arith == MPS_ARITH_EXACT, h->cap, h->stream, h->ppe.lp.tensor_cores);
    h->ppe.lp.s_ready = false;
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaGetLastError());
    if (loss_first) *loss_first = first;
    if (loss_last) *loss_last = last;
    return MPS_OK;
}

// Run the network forward on the last PPE system with the 64 -> 64 layers in
// FP32 on the CUDA cores and with BF16 activations on the tensor cores,
// report the largest difference of the factor's entries relative to the
// largest entry, and use the tensor cores for inference from now on when
// `enable` is set.
extern "C" mps_status mps_precond_tensor_cores(mps_handle* h, int enable, double* max_rel_diff) {
    mps_status s = need_snapshot(h, true);
    if (s != MPS_OK) return s;
    CK(cudaSetDevice(h->dev));
    const LpSystem L = ppe_lp_system(h->ppe, stage_args(h));
    const bool exact = h->opt.arith == MPS_ARITH_EXACT;
    const size_t ng = (size_t)h->cap * LP_GW, nd = h->cap;
    std::vector<float> g0(ng), d0(nd), g1(ng), d1(nd);
    lp_build_stencil(h->ppe.lp, L, h->cap, h->stream);  // this system's stencil
    for (int pass = 0; pass < 2; pass++) {
        lp_forward(h->ppe.lp, L, exact, h->cap, h->stream, pass == 1);
        CK(cudaMemcpyAsync(pass ? g1.data() : g0.data(), h->ppe.lp.gval, ng * 4, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaMemcpyAsync(pass ? d1.data() : d0.data(), h->ppe.lp.gdiag, nd * 4, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        CK(cudaGetLastError());
    }
    double mx = 0.0, md = 0.0;
    for (size_t k = 0; k < ng; k++) {
        mx = std::max(mx, (double)std::fabs(g0[k]));
        md = std::max(md, (double)std::fabs(g0[k] - g1[k]));
    }
    for (size_t k = 0; k < nd; k++) {
        mx = std::max(mx, (double)std::fabs(d0[k]));
        md = std::max(md, (double)std::fabs(d0[k] - d1[k]));
    }
    if (max_rel_diff) *max_rel_diff = mx > 0.0 ? md / mx : md;
    h->ppe.lp.tensor_cores = enable != 0;
    lp_forward(h->ppe.lp, L, exact, h->cap, h->stream, h->ppe.lp.tensor_cores);
    CK(cudaStreamSynchronize(h->stream));
    h->ppe.lp.s_ready = false;  // the next step evaluates the network with the chosen layers
    drop_graphs(h);
    Scalars sc;
    return read_status(h, &sc);
}

extern "C" mps_status mps_precond_train_tensor_cores(mps_handle* h, int enable) {
    mps_status s = need_semi(h);
    if (s != MPS_OK) return s;
    h->ppe.lp.train_tensor_cores = enable != 0;
    return MPS_OK;
}

extern "C" mps_status mps_ppe_snapshot(mps_handle* h, float* pos4, float* n, uint32_t* id, uint32_t* is_row,
                                       double* diag, uint32_t* count) {
    mps_status s = need_semi(h);
    if (s != MPS_OK) return s;
    if (!h->ppe.have_snapshot) {
        h->err = "no PPE system assembled yet";
        return MPS_ERR_INVALID;
    }
    CK(cudaSetDevice(h->dev));
    Scalars sc;
    if (counts(h, &sc) != MPS_OK) return MPS_ERR_CUDA;
    const size_t np = sc.np;
    cudaStream_t st = h->stream;
    if (pos4) CK(cudaMemcpyAsync(pos4, h->ppe.pos_snap, np * 16, cudaMemcpyDeviceToHost, st));
    if (n) CK(cudaMemcpyAsync(n, h->ppe.n_snap, np * 4, cudaMemcpyDeviceToHost, st));
    if (id) CK(cudaMemcpyAsync(id, h->ppe.id_snap, np * 4, cudaMemcpyDeviceToHost, st));
    if (diag) CK(cudaMemcpyAsync(diag, h->ppe.diag64, np * 8, cudaMemcpyDeviceToHost, st));
    if (is_row) {
        CK(cudaMemcpyAsync(is_row, h->ppe.rlen, np * 4, cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    if (is_row)
        for (size_t k = 0; k < np; k++) is_row[k] = is_row[k] != PPE_DIRICHLET ? 1u : 0u;
    if (count) *count = (uint32_t)np;
    return MPS_OK;
}

extern "C" mps_status mps_ppe_stencil(mps_handle* h, uint32_t* row_start, uint32_t* cols, float* weights,
                                      uint64_t max_entries, uint64_t* nnz) {
    mps_status s = need_semi(h, true);
    if (s != MPS_OK) return s;
    if (!h->ppe.have_snapshot) {
        h->err = "no PPE system assembled yet";
        return MPS_ERR_INVALID;
    }
    CK(cudaSetDevice(h->dev));
    Scalars sc;
    if (counts(h, &sc) != MPS_OK) return MPS_ERR_CUDA;
    const int rc = ppe_export_stencil(h->ppe, sc.np, row_start, cols, weights, max_entries, nnz, h->stream);
    if (rc == MPS_ERR_CAPACITY) h->err = "the stencil has more entries than max_entries";
    return (mps_status)rc;
}

extern "C" const char* mps_stage_name(int k) { return (k >= 0 && k < ST_COUNT) ? kStageNames[k] : ""; }

extern "C" mps_status mps_profile_steps(mps_handle* h, int nsteps, double* stage_ms, int max_stages,
                                        int* nstages) {
    if (!h || nsteps < 0 || !stage_ms) return MPS_ERR_INVALID;
    CK(cudaSetDevice(h->dev));
    for (int k = 0; k < max_stages; k++) stage_ms[k] = 0.0;
    if (nstages) *nstages = ST_COUNT;
    for (int s = 0; s < nsteps; s++) {
        h->prof_on = true;
        h->prof_used = 0;
        begin_step(h);
        enqueue_step(h);
        mark(h, -1);
        h->prof_on = false;
        CK(cudaStreamSynchronize(h->stream));
        CK(cudaGetLastError());
        for (size_t k = 0; k + 1 < h->prof_used; k++) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, h->prof_ev[k], h->prof_ev[k + 1]);
            const int t = h->prof_tag[k];
            if (t >= 0 && t < max_stages) stage_ms[t] += ms;
        }
    }
    return read_status(h, nullptr);
}

// Autotuner: the block size of the particle-stage kernels (64, 128, 256),
// and for the persistent PPE solver the grid shape (1024, 512 or 256
// threads per block, 1024 threads per SM) and its form (stored weights,
// weights recomputed from positions, or stored weights with the pipelined
// single-reduction PCG), each timed with CUDA events over `steps` steps of
// the handle's own scene; the fastest is kept.  The scene advances by the
// steps taken.
extern "C" mps_status mps_autotune(mps_handle* h, int steps, mps_tune_report* rep) {
    if (!h || steps < 1) return MPS_ERR_INVALID;
    CK(cudaSetDevice(h->dev));
    mps_tune_report r;
    memset(&r, 0, sizeof r);
    std::vector<double> ms(32);
    int nst = 0;
    const int stage_cand[3] = {64, 128, 256};
    double best = 1e300;
    int best_t = h->stage_threads;
    for (int c = 0; c < 3; c++) {
        h->stage_threads = stage_cand[c];
        drop_graphs(h);
        mps_status st = mps_profile_steps(h, steps, ms.data(), 32, &nst);
        if (st != MPS_OK) return st;
        const double t = (ms[ST_VISC] + ms[ST_COLLISION] + ms[ST_PND] + ms[ST_DASH]) / steps;
        r.stage_ms[c] = (float)t;
        if (t < best) {
            best = t;
            best_t = stage_cand[c];
        }
    }
    h->stage_threads = best_t;
    r.stage_threads = best_t;
    r.ppe_threads = h->ppe.threads;
    if (h->opt.method == MPS_METHOD_SEMI_IMPLICIT) {
        // forms: 0 stored weights, 1 recomputed weights, 2 stored weights
        // with the pipelined (single-reduction) PCG; the learned and batched
        // solvers have no pipelined form
        const int ppe_cand[3] = {1024, 512, 256};
        const bool learned = h->opt.precond == MPS_PRECOND_LEARNED && h->ppe.lp.ready;
        const int nforms = (learned || h->nscenes) ? 2 : 3;
        // form 3: the compact layout (single scenes, diagonal scaling)
        const bool compact_ok = h->ppe.c16_ready && !h->nscenes && (!learned || h->ppe.sp_ent != nullptr);
        best = 1e300;
        int best_p = h->ppe.threads;
        bool best_sw = h->ppe.stored_weights, best_pipe = h->ppe.pipelined, best_c16 = h->ppe.c16;
        for (int k = 0; k < 3; k++) r.ppe_compact_ms[k] = -1.f;
        for (int c = 0; c < 12; c++) {
            const int form = c / 3;
            if (form >= nforms && form != 3) {
                r.ppe_ms[c] = -1.f;
                continue;
            }
            if (form == 3 && !compact_ok) continue;
            const bool pipe = form == 2;
            const int threads = ppe_cand[c % 3];
            if (ppe_set_threads(h->ppe, threads) != MPS_OK) {
                if (form < 3) r.ppe_ms[c] = -1.f;  // the device cannot hold this shape
                continue;
            }
            h->ppe.stored_weights = form != 1;
            h->ppe.pipelined = pipe;
            set_compact(h, form == 3);
            drop_graphs(h);
            double tot = 0.0;
            for (int k = 0; k < steps; k++) {
                mps_status st = mps_profile_steps(h, 1, ms.data(), 32, &nst);
                if (st != MPS_OK) return st;
                tot += ms[ST_PPE_SOLVE];
            }
            const double t = tot / steps;
            if (form < 3) r.ppe_ms[c] = (float)t;
            else r.ppe_compact_ms[c % 3] = (float)t;
            if (t < best) {
                best = t;
                best_p = threads;
                best_sw = form != 1;
                best_pipe = pipe;
                best_c16 = form == 3;
            }
        }
        ppe_set_threads(h->ppe, best_p);
        h->ppe.stored_weights = best_sw;
        h->ppe.pipelined = best_pipe;
        set_compact(h, best_c16);
        r.ppe_threads = best_p;
        r.ppe_stored_weights = best_sw ? 1 : 0;
        r.ppe_pipelined = best_pipe ? 1 : 0;
        r.ppe_compact = best_c16 ? 1 : 0;
    }
    drop_graphs(h);
    if (rep) *rep = r;
    return MPS_OK;
}

extern "C" mps_status mps_apply_tuning(mps_handle* h, const mps_tune_report* r) {
    if (!h || !r) return MPS_ERR_INVALID;
    if (r->stage_threads != 64 && r->stage_threads != 128 && r->stage_threads != 256) return MPS_ERR_INVALID;
    CK(cudaSetDevice(h->dev));
    CK(cudaStreamSynchronize(h->stream));
    h->stage_threads = r->stage_threads;
    if (h->opt.method == MPS_METHOD_SEMI_IMPLICIT) {
        const bool learned = h->opt.precond == MPS_PRECOND_LEARNED && h->ppe.lp.ready;
        if (r->ppe_compact) {
            if (h->nscenes) {
                h->err = "the compact PPE layout is for single scenes";
                return MPS_ERR_INVALID;
            }
            int e = ppe_c16_enable(h->ppe, &h->err);
            if (e == MPS_OK && h->opt.precond == MPS_PRECOND_LEARNED) e = ppe_c16_learned_enable(h->ppe, &h->err);
            if (e != MPS_OK) return (mps_status)e;
        }
        if (r->ppe_pipelined && (learned || h->nscenes)) {
            h->err = "the pipelined PCG is for single scenes with diagonal scaling";
            return MPS_ERR_INVALID;
        }
        if (ppe_set_threads(h->ppe, r->ppe_threads) != MPS_OK) {
            h->err = "the device cannot hold that PPE block size";
            return MPS_ERR_INVALID;
        }
        h->ppe.stored_weights = r->ppe_stored_weights != 0;
        h->ppe.pipelined = r->ppe_pipelined != 0;
        set_compact(h, r->ppe_compact != 0);
    }
    drop_graphs(h);
    return MPS_OK;
}

// ---------------------------------------------------------------- free surface
extern "C" mps_status mps_surface_case_table(uint8_t* ntri, int8_t* tri) {
    if (!ntri || !tri) return MPS_ERR_INVALID;
    mc_build_table(ntri, reinterpret_cast<int8_t(*)[16]>(tri));
    return MPS_OK;
}

static mps_status need_surface(mps_handle* h) {
    if (!h) return MPS_ERR_INVALID;
    if (!h->surf.ready) {
        h->err = "call mps_surface_setup first";
        return MPS_ERR_INVALID;
    }
    return MPS_OK;
}

extern "C" mps_status mps_surface_setup(mps_handle* h, const mps_surface_grid* g, uint32_t max_triangles) {
    if (!h || !g || max_triangles == 0) return MPS_ERR_INVALID;
    if (h->nscenes) {
        h->err = "surfaces are extracted from single-scene handles";
        return MPS_ERR_INVALID;
    }
    CK(cudaSetDevice(h->dev));
    SurfaceGrid sg;
    sg.nx = g->nx;
    sg.ny = g->ny;
    sg.nz = g->nz;
    sg.ox = g->origin[0];
    sg.oy = g->origin[1];
    sg.oz = g->origin[2];
    sg.hx = g->spacing[0];
    sg.hy = g->spacing[1];
    sg.hz = g->spacing[2];
    int e = surface_setup(h->surf, sg, max_triangles, h->stream, &h->err);
    if (e != MPS_OK) return (mps_status)e;
    surface_enqueue_iso(h->surf, stage_args(h), h->cap, h->stream);
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaGetLastError());
    uint32_t bits[2];
    CK(cudaMemcpy(bits, h->surf.ntri, 8, cudaMemcpyDeviceToHost));
    memcpy(&h->surf.iso, &bits[1], 4);
    return MPS_OK;
}

extern "C" mps_status mps_surface_extract_async(mps_handle* h) {
    mps_status s = need_surface(h);
    if (s != MPS_OK) return s;
    CK(cudaSetDevice(h->dev));
    surface_enqueue_extract(h->surf, stage_args(h), h->stream);
    CK(cudaGetLastError());
    return MPS_OK;
}

extern "C" mps_status mps_surface_extract(mps_handle* h, uint32_t* ntri) {
    mps_status s = mps_surface_extract_async(h);
    if (s != MPS_OK) return s;
    uint32_t n = 0;
    CK(cudaMemcpyAsync(&n, h->surf.ntri, 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (ntri) *ntri = n;
    if (n > h->surf.max_tri) {
        h->err = "the surface has more triangles than the buffer holds (" + std::to_string(n) + ")";
        return MPS_ERR_CAPACITY;
    }
    return MPS_OK;
}

extern "C" mps_status mps_surface_get(mps_handle* h, float* pos9, float* nrm9, uint32_t max_triangles,
                                      uint32_t* ntri) {
    mps_status s = need_surface(h);
    if (s != MPS_OK) return s;
    CK(cudaSetDevice(h->dev));
    uint32_t n = 0;
    CK(cudaMemcpyAsync(&n, h->surf.ntri, 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (ntri) *ntri = n;
    uint32_t m = n < h->surf.max_tri ? n : h->surf.max_tri;
    m = m < max_triangles ? m : max_triangles;
    if (m && pos9) CK(cudaMemcpyAsync(pos9, h->surf.tri_pos, (size_t)m * 36, cudaMemcpyDeviceToHost, h->stream));
    if (m && nrm9) CK(cudaMemcpyAsync(nrm9, h->surf.tri_nrm, (size_t)m * 36, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return MPS_OK;
}

extern "C" mps_status mps_surface_vertex_values(mps_handle* h, float* values, float* iso) {
    mps_status s = need_surface(h);
    if (s != MPS_OK) return s;
    CK(cudaSetDevice(h->dev));
    const SurfaceGrid& g = h->surf.g;
    if (values)
        CK(cudaMemcpyAsync(values, h->surf.vn, (size_t)g.nx * g.ny * g.nz * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (iso) *iso = h->surf.iso;
    return MPS_OK;
}

extern "C" mps_status mps_surface_write_stl(mps_handle* h, const char* path) {
    mps_status s = need_surface(h);
    if (s != MPS_OK) return s;
    if (!path) return MPS_ERR_INVALID;
    uint32_t n = 0;
    s = mps_surface_get(h, nullptr, nullptr, 0, &n);
    if (s != MPS_OK) return s;
    const uint32_t m = n < h->surf.max_tri ? n : h->surf.max_tri;
    std::vector<float> p((size_t)m * 9), q((size_t)m * 9);
    s = mps_surface_get(h, p.data(), q.data(), m, &n);
    if (s != MPS_OK) return s;
    FILE* f = fopen(path, "wb");
    if (!f) return MPS_ERR_IO;
    char header[80];
    memset(header, 0, sizeof header);
    snprintf(header, sizeof header, "MPS free surface, %u triangles", m);
    fwrite(header, 1, 80, f);
    fwrite(&m, 4, 1, f);
    for (uint32_t t = 0; t < m; t++) {
        float rec[12];
        for (int d = 0; d < 3; d++) rec[d] = (q[9 * t + d] + q[9 * t + 3 + d] + q[9 * t + 6 + d]) / 3.f;
        for (int k = 0; k < 9; k++) rec[3 + k] = p[9 * (size_t)t + k];
        fwrite(rec, 4, 12, f);
        const uint16_t attr = 0;
        fwrite(&attr, 2, 1, f);
    }
    const bool ok = fclose(f) == 0;
    return ok ? MPS_OK : MPS_ERR_IO;
}

extern "C" mps_status mps_get_normal_ids(mps_handle* h, uint32_t* normal_id) {
    if (!h || !normal_id) return MPS_ERR_INVALID;
    CK(cudaSetDevice(h->dev));
    CK(cudaMemcpyAsync(normal_id, h->normal_id_of, h->np0 * sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return MPS_OK;
}

extern "C" mps_status mps_get_stream(mps_handle* h, void** stream) {
    if (!h || !stream) return MPS_ERR_INVALID;
    *stream = (void*)h->stream;
    return MPS_OK;
}

extern "C" mps_status mps_write_case(mps_handle* h, const char* path, int format) {
    if (!h || !path || (format != 0 && format != 1)) return MPS_ERR_INVALID;
    uint32_t np = 0;
    mps_status s = mps_get_counts(h, &np, nullptr, nullptr, nullptr);
    if (s != MPS_OK) return s;
    std::vector<uint32_t> id(np), type(np);
    std::vector<float> pos(3 * (size_t)np), vel(3 * (size_t)np), pr(np);
    s = mps_get_state(h, id.data(), type.data(), pos.data(), vel.data(), pr.data(), nullptr, MPS_ORDER_SORTED);
    if (s != MPS_OK) return s;
    return (mps_status)write_case_text(path, format, np, id.data(), type.data(), pos.data(), vel.data(), pr.data());
}

// MPS_GPU_EXPL::mps_cal (MPS_CAL_expl_v1.0/MPS_GPU_EXPL.cpp:216-272): output
// whenever time - threshold >= 0, threshold += tout; then a step.
extern "C" mps_status mps_run(mps_handle* h, const char* out_dir) {
    if (!h) return MPS_ERR_INVALID;
    if (h->nscenes) {
        h->err = "mps_run drives a single scene; step a batch with mps_batch_step";
        return MPS_ERR_INVALID;
    }
    float threshold = 0.0f;
    int count = 0;
    for (;;) {
        Scalars s;
        mps_status st = read_status(h, &s);
        if (st != MPS_OK) return st;
        if (!(s.time < h->prm.tt)) break;
        if (s.time - threshold >= 0.0f) {
            if (out_dir) {
                char path[4096];
                snprintf(path, sizeof path, "%s/%04d.out", out_dir, count);
                st = mps_write_case(h, path, h->opt.method == MPS_METHOD_EXPLICIT ? 0 : 1);
                if (st != MPS_OK) return st;
            }
            threshold += h->prm.tout;
            count++;
        }
        st = step_async(h, 1);
        if (st != MPS_OK) return st;
    }
    return MPS_OK;
}

// ---------------------------------------------------------------- primitive
extern "C" mps_status mps_cell_sort_dev(const float* pos4_dev, uint32_t n, const mps_grid* gg, uint32_t* perm_dev,
                                        uint32_t* cell_of_dev, uint32_t* start_dev, uint32_t* end_dev,
                                        uint32_t* n_in_grid_dev, void* stream) {
    if (!gg || (n && (!pos4_dev || !perm_dev || !cell_of_dev)) || !start_dev || !end_dev || !n_in_grid_dev)
        return MPS_ERR_INVALID;
    if (gg->ncells == 0 || gg->ncells >= 0x7fffffffu) return MPS_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    Grid g;
    g.left = gg->left;
    g.back = gg->back;
    g.bottom = gg->bottom;
    g.cell_size = gg->cell_size;
    g.cdx = gg->cdx;
    g.cdy = gg->cdy;
    g.cdz = gg->cdz;
    g.sheet = gg->cdx * gg->cdy;
    g.ncells = gg->ncells;
    g.dim = gg->dim;
    g.cell_yz = gg->cell_yz > 0.f ? gg->cell_yz : gg->cell_size;
    g.reach = walk_reach(g.cell_size, g.cell_yz);
    g.base = 0;
    const uint32_t tiles = sort_tiles(n > 0 ? n : 1);
    SortScratch s;
    s.tiles = tiles;
    void* blk = nullptr;
    const size_t nk = (size_t)(n > 0 ? n : 1);
    const size_t bytes = 4 * nk * sizeof(uint32_t) + (size_t)SORT_RADIX * tiles * sizeof(uint32_t) +
                         ((size_t)g.ncells + 1) * sizeof(uint32_t) + sizeof(uint32_t) + 256;
    if (cudaMalloc(&blk, bytes) != cudaSuccess) return MPS_ERR_CUDA;
    uint32_t* b = (uint32_t*)blk;
    s.keys[0] = b;
    s.vals[0] = b + nk;
    s.keys[1] = b + 2 * nk;
    s.vals[1] = b + 3 * nk;
    s.hist = b + 4 * nk;
    uint32_t* cs = s.hist + (size_t)SORT_RADIX * tiles;
    uint32_t* n_dev = cs + g.ncells + 1;
    cudaMemcpyAsync(n_dev, &n, sizeof n, cudaMemcpyHostToDevice, st);
    launch_cell_keys_plain((const float4*)pos4_dev, n, g, s.keys[0], s.vals[0], st);
    const int r = launch_radix_sort(s, n_dev, sort_passes(g.ncells), n, st);
    launch_cell_start_plain(s.keys[r], n, g, cs, n_in_grid_dev, st);
    if (n) {
        cudaMemcpyAsync(perm_dev, s.vals[r], n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(cell_of_dev, s.keys[r], n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st);
    }
    launch_cell_end_from_start(cs, g.ncells, start_dev, end_dev, st);
    cudaError_t e = cudaStreamSynchronize(st);
    cudaFree(blk);
    if (e != cudaSuccess || cudaGetLastError() != cudaSuccess) return MPS_ERR_CUDA;
    return MPS_OK;
}
