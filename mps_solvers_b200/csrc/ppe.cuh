// ppe.cuh -- pressure Poisson equation of the semi-implicit step.
//
// MPS_CPU::buildPoisson + solvePoisson + pressCorr (MPS_CAL_v4.0/MPS_CPU.cpp:619-743):
// for a particle i of type != 2 with n_i >= beta n0 (not Dirichlet)
//   A_ij = w(r_ij; rlap)            for neighbours j of type != 2, not Dirichlet
//   A_ii = -sum_j w(r_ij; rlap) - rho lambda alpha n0 / (2 d dt^2)   (all type != 2 neighbours)
//   b_i  = lambda rho / (2 d dt_max^2) (n0 - n_i)
// Dirichlet rows (n_i < beta n0 or type 2) are identity rows with b = 0, so
// their solution is 0 and they are left out of the solve.  Then p = max(x, 0).
//
// Storage: the neighbour stencil of each row (column indices, in sliced-ELL
// order) and the diagonal in double; the off-diagonal weights are recomputed
// from the float positions in every matrix product with the same function
// the assembly used (matrix-free in the weights).
#pragma once
#include <cstdint>
#include <string>
#include <cuda_runtime.h>

#include "../../include/mps_capi.h"
#include "learned.cuh"
#include "physics.cuh"

namespace mpsb {

constexpr uint32_t PPE_W = 512;        // stride: 2x the 256 lattice neighbours within 4 l0
constexpr uint32_t PPE_DIRICHLET = 0xffffffffu;
constexpr int PPE_THREADS = 1024;
constexpr int PPE_PARTS = 4;           // FP64 partial sums per block
constexpr uint32_t SELL_C = 8;         // rows per sliced-ELL slice
constexpr int PPE_SMEM_CHUNKS = 6;     // 8-byte layout: most 1 KB chunks a warp keeps in shared memory
constexpr uint32_t PPE_MAX_SCENES = 256;  // scenes of a batch the solver holds in shared memory

// PPE constants of one scene of a batch (MPS_CAL_v4.0/MPS_CPU.cpp:619-650)
struct PpeScene {
    double n0, beta, b_tmp, rho_lambda_alpha_n0;
};

struct PpeWork {
    bool ready = false;
    uint32_t cap = 0;
    int blocks = 0;                    // co-resident blocks of the persistent solver
    int threads = PPE_THREADS;         // its block size (1024 / threads blocks per SM)
    int sms = 0;
    uint32_t* cols = nullptr;          // cap * PPE_W
    float* wrm = nullptr;              // their weights
    uint32_t* rlen = nullptr;          // off-diagonal count, PPE_DIRICHLET for Dirichlet rows
    double* diag64 = nullptr;
    float* diag32 = nullptr;
    float* inv_diag = nullptr;
    double* b64 = nullptr;
    double* x64 = nullptr;
    float *r = nullptr, *q = nullptr, *qp = nullptr;
    float2* zp[2] = {nullptr, nullptr};  // (z, p) per row: current and next
    double* part = nullptr;            // blocks * PPE_PARTS
    double* result = nullptr;          // PPE_PARTS grid totals
    uint32_t* rowlist = nullptr;       // non-Dirichlet rows in particle order
    uint32_t* tilecnt = nullptr;
    uint32_t* nrows = nullptr;
    uint32_t* sell_off = nullptr;      // slice offsets (exclusive scan of 32 * width)
    uint32_t* sell_cols = nullptr;
    float* sell_w = nullptr;           // the entries' weights, same layout
    bool stored_weights = true;        // SpMV reads sell_w (else recomputes from positions)
    bool pipelined = false;            // single-reduction pipelined PCG (diagonal scaling)
    bool write_pressure = true;        // the solve ends by writing p = max(x, 0) (the PPE; not the viscosity)
    uint32_t l2_keep_entries = 0xFFFFFFFFu;  // matrix entries kept in L2 across iterations (all: no hints)
    // vectors of the pipelined solver
    float *pu = nullptr, *pw = nullptr, *pz = nullptr, *pq = nullptr, *ps = nullptr, *pp = nullptr;
    float* pm[2] = {nullptr, nullptr};
    unsigned* bar = nullptr;           // [0] arrival count, [1] generation
    // learned preconditioner (set up on first use)
    LearnedWork lp;
    // state at the last assembly (the system the network and its training see)
    float4* pos_snap = nullptr;
    float* n_snap = nullptr;
    uint32_t* id_snap = nullptr;
    bool have_snapshot = false;
    double n0_64 = 0.0, lambda64 = 0.0, alpha64 = 0.0;
    cudaError_t launch_err = cudaSuccess;  // of the last cooperative launch
    // batch: per-scene constants, scene of each row, per-scene results
    uint32_t nscenes = 0;
    PpeScene* scenes = nullptr;
    uint32_t* row_scene = nullptr;
    double* bpart = nullptr;           // blocks * 3 * nscenes
    double* bresult = nullptr;         // 3 * nscenes
    int* scene_iters = nullptr;
    int* scene_outer = nullptr;
    double* scene_relres = nullptr;
    // compact layout (ppe_compact.cu): rows numbered 0..R-1 in row-list
    // order, slices of 4 rows with 8 lanes per row, 16-bit column codes
    // relative to the slice, FP32 weights; single scenes, diagonal scaling
    bool c16 = false;                  // the solve uses this layout
    bool c16_ready = false;            // its buffers exist
    int c16_smem_chunks = 8;           // chunks per warp held in shared memory across iterations
    size_t c16_cap_chunks = 0;
    uint32_t* cpos = nullptr;          // compact row of each particle (rows only)
    uint32_t* c16_width = nullptr;     // chunks per slice, then (scanned) the slices' first chunk
    uint16_t* c16_codes = nullptr;     // 128 codes per chunk (column - 4 * slice + 32768; 65535: escaped)
    float* c16_w = nullptr;            // 128 weights per chunk
    uint32_t* c16_side = nullptr;      // compact column of an escaped entry (same layout)
    uint32_t* c16_esc = nullptr;       // escaped entries of the last pack
    double *cb64 = nullptr, *cx64 = nullptr, *cdiag64 = nullptr;
    float *cdiag32 = nullptr, *cinv_diag = nullptr, *cr = nullptr, *cq = nullptr;
    float2* czp[2] = {nullptr, nullptr};
    // the learned preconditioner: S' = D^-1/2 S D^-1/2 (S the symmetric form
    // in LearnedWork, kept by GEO index, rebuilt every precond_every steps)
    // packed for the current rows every step (layout: ppe_device.cuh), one
    // product fused into the residual update of every PCG iteration; its
    // columns are compact positions for the compact solver and particle
    // indices for the 8-byte and batch solvers
    bool c16_learned = false;          // the compact solve applies S'
    int precond_every = 40;            // steps between network evaluations
    uint32_t* sp_off = nullptr;        // first entry of every 32-row slice (widths, then scanned)
    uint32_t* sp_ent = nullptr;        // off-diagonal entries: column - own column (16 bits) << 16 | BF16 value
    float* sp_diag = nullptr;          // the diagonal, per row position
    float* cr2 = nullptr;              // second residual buffer of the compact solver's fused update
    float2* rq[2] = {nullptr, nullptr};  // the 8-byte and batch solvers' (r, q) pairs, current and next
    size_t sp_cap_chunks = 0;
    const uint32_t* index_of_id = nullptr;  // the handle's GEO index -> sorted position
    bool build_net = true;             // this step evaluates the network (learned preconditioner)
    uint64_t net_steps = 0;            // steps since the handle was created
};

// The learned preconditioner re-evaluates its network every precond_every
// steps (and whenever its form has not been built): decide for the next
// step, count it, and return the decision.
inline bool ppe_begin_step(PpeWork& w) {
    w.build_net = !w.lp.s_ready || w.precond_every <= 1 || (w.net_steps % (uint64_t)w.precond_every) == 0;
    w.net_steps++;
    return w.build_net;
}

int ppe_setup(PpeWork& w, uint32_t cap, const Grid& g, const Phys& P, const mps_params& prm, cudaStream_t st,
              std::string* err);
// the per-scene tables of a batch (after ppe_setup)
int ppe_setup_batch(PpeWork& w, const PpeScene* scenes, uint32_t nscenes, cudaStream_t st, std::string* err);
// assembly, row list and sliced-ELL layout (and, with the learned
// preconditioner, its stencil and network forward); returns the kernels enqueued
int ppe_enqueue_setup(PpeWork& w, const StageArgs& a, const mps_options& opt, uint32_t cap, cudaStream_t st);
// the system the network works on, from the last assembly
LpSystem ppe_lp_system(const PpeWork& w, const StageArgs& a);
int ppe_enable_learned(PpeWork& w, std::string* err);
// the persistent solve and p = max(x, 0); returns the kernels enqueued
int ppe_enqueue_solve(PpeWork& w, const StageArgs& a, const mps_options& opt, uint32_t cap, cudaStream_t st);
// Crank-Nicolson viscosity (MPS_CPU_IMPL::visCrankNicolson) for velocity
// component c on a PpeWork of its own: assembly, rows, pack, the persistent
// PCG, and u_c = x, x_c += dt u_c for the fluid.  Returns the launches.
int ppe_enqueue_cn(PpeWork& w, const StageArgs& a, const mps_options& opt, int c, double n0, double lambda,
                   uint32_t cap, cudaStream_t st);
void ppe_free(PpeWork& w);
// the stored off-diagonal entries of the last assembly as per-row lists in
// particle order (host arrays; cols/wts may be NULL to size them first)
int ppe_export_stencil(const PpeWork& w, uint32_t np, uint32_t* row_start, uint32_t* cols, float* wts,
                       uint64_t max_entries, uint64_t* nnz, cudaStream_t st);
// The compact 16-bit layout and its persistent solver (ppe_compact.cu):
// buffers, the pack after the row list, the solve with p = max(x, 0), the
// escaped-entry count of the last pack, and the stencil export.
int ppe_c16_enable(PpeWork& w, std::string* err);
int ppe_c16_enqueue_pack(PpeWork& w, const StageArgs& a, uint32_t cap, cudaStream_t st);
int ppe_c16_enqueue_solve(PpeWork& w, const StageArgs& a, const mps_options& opt, uint32_t cap, cudaStream_t st);
int ppe_c16_export(const PpeWork& w, uint32_t np, const uint32_t* d_row_start, uint32_t* d_cols, float* d_w,
                   cudaStream_t st);
void ppe_c16_free(PpeWork& w);
// the learned S': its buffers (ppe_sp_enable; the compact solver's second
// residual buffer too with ppe_c16_learned_enable), and its per-step pack
// from the symmetric form kept by GEO index, after the row list (and, for
// the compact columns, after ppe_c16_enqueue_pack)
int ppe_sp_enable(PpeWork& w, std::string* err);
int ppe_c16_learned_enable(PpeWork& w, std::string* err);
int ppe_sp_enqueue_pack(PpeWork& w, const StageArgs& a, uint32_t cap, cudaStream_t st, bool by_particle);
// the persistent solver's block size (256, 512 or 1024; 1024 threads per SM
// either way); MPS_ERR_INVALID when the device cannot hold that shape
int ppe_set_threads(PpeWork& w, int threads);

// FP64 particle number density of every particle (initialisation of the
// semi-implicit method: n0 and lambda in double, MPS_CAL_v4.0/MPS.cpp:305-361)
void launch_pnd64(const StageArgs& a, double* n64, uint32_t cap, cudaStream_t st);
// out[0] = n0, out[1] = lambda (double), over the particles [lo, hi) (all: 0, ~0u)
void launch_n0_lambda64(const StageArgs& a, const double* n64, double* out, cudaStream_t st, uint32_t lo = 0,
                        uint32_t hi = 0xffffffffu);

}  // namespace mpsb
