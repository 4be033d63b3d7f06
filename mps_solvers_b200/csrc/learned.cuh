// learned.cuh -- learned sparse-factor preconditioner of the PPE.
//
// M^-1 = D^-1/2 G^T G D^-1/2 with D = diag(-A) and G lower triangular (in
// the sorted particle order) on the non-Dirichlet rows, with a positive
// diagonal: SPD for any network output.  G's pattern is each row's
// neighbours within r0 (the particle-number-density stencil) that come
// before it, plus the diagonal.  The entries come from a small
// message-passing network over that stencil:
//
//   edge features e_ij (7): dx/r0, dy/r0, dz/r0, |r|/r0, w(r; r0)/w_ref,
//                           n_i/n0, [j is a wall particle]
//   pass 1: a1_i = mean_j GELU(W1e e_ij + b1)            (64)
//            h1_i = GELU(V1 a1_i + c1)                      (64)
//   pass 2: a2_i = mean_j GELU(W2e e_ij + U2 h1_j + b2)   (64)
//            h2_i = GELU(V2 a2_i + c2) + h1_i               (64)
//   readout: G_ij = om . GELU(Re e_ij + Ra h2_i + Rb h2_j + br)   (j < i)
//            G_ii = softplus(dl . h2_i + bd) + GMIN
//
// GELU is the tanh form.  Weights are stored in BF16 for the kernels and in
// FP32 (master copy, Adam moments) for training; every sum accumulates in
// FP32.  Training minimises Kaporin's condition number of the preconditioned
// matrix, beta = (tr(M) / n) / det(M)^(1/n) with M = G Ahat G^T and
// Ahat = D^-1/2 (-A) D^-1/2, through
//   L = log(z^T M z / n) - (2 / n) sum_i log G_ii     (= log beta + const),
// with a Rademacher probe z (Hutchinson's trace estimate) on PPE systems the
// solver produced.  L is invariant to the scale of G, and over a fixed
// sparsity pattern its minimiser is the factorized sparse approximate inverse
// (Kolotilina and Yeremin, 1993); CG's iteration bound follows beta
// (Kaporin, 1994).
//
// The solvers apply the symmetric first-order form S of G^T G (below),
// scaled to S' = D^-1/2 S D^-1/2: one product a PCG iteration, fused into
// the residual update.
#pragma once
#include <cstdint>
#include <string>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "physics.cuh"

namespace mpsb {

constexpr int LP_H = 64;    // hidden width
constexpr int LP_F = 7;     // edge features
constexpr int LP_GW = 64;   // stencil stride: 2x the 32 lattice neighbours within r0
constexpr float LP_GMIN = 1e-3f;

// parameter offsets (floats) in the flat parameter vector
enum : int {
    LP_W1E = 0,                        // [64][7]
    LP_B1 = LP_W1E + LP_H * LP_F,      // [64]
    LP_V1 = LP_B1 + LP_H,              // [64][64]
    LP_C1 = LP_V1 + LP_H * LP_H,       // [64]
    LP_W2E = LP_C1 + LP_H,             // [64][7]
    LP_U2 = LP_W2E + LP_H * LP_F,      // [64][64]
    LP_B2 = LP_U2 + LP_H * LP_H,       // [64]
    LP_V2 = LP_B2 + LP_H,              // [64][64]
    LP_C2 = LP_V2 + LP_H * LP_H,       // [64]
    LP_RE = LP_C2 + LP_H,              // [64][7]
    LP_RA = LP_RE + LP_H * LP_F,       // [64][64]
    LP_RB = LP_RA + LP_H * LP_H,       // [64][64]
    LP_BR = LP_RB + LP_H * LP_H,       // [64]
    LP_OM = LP_BR + LP_H,              // [64]
    LP_DL = LP_OM + LP_H,              // [64]
    LP_BD = LP_DL + LP_H,              // [1]
    LP_NPARAM = LP_BD + 1
};

struct LearnedWork {
    bool ready = false;
    bool tensor_cores = false;       // inference forward on tcgen05 (set after a self-check)
    bool train_tensor_cores = false; // training's 64 -> 64 products on tcgen05 (BF16 operands)
    uint32_t cap = 0;
    // parameters
    float* w32 = nullptr;            // FP32 master
    __nv_bfloat16* w16 = nullptr;    // BF16 copy used by the kernels
    float* grad = nullptr;
    float* adam_m = nullptr;
    float* adam_v = nullptr;
    int adam_t = 0;
    // stencil (neighbours within r0 among non-Dirichlet rows)
    uint32_t* scols = nullptr;       // cap * LP_GW, ascending index
    uint32_t* scnt = nullptr;        // cap
    uint32_t* nlow = nullptr;        // cap: entries with j < i (they come first)
    // factor G, row i: gdiag[i], glow[i*GW + t] = G_ij for the first nlow
    // entries, gup[i*GW + t] = G_ji for the later (j > i) entries
    float* gdiag = nullptr;
    float* gval = nullptr;
    // node activations (cap * 64)
    float *a1 = nullptr, *pre1 = nullptr, *h1 = nullptr, *uh1 = nullptr, *a2 = nullptr, *pre2 = nullptr,
          *h2 = nullptr, *ra = nullptr, *rb = nullptr;
    float* dgpre = nullptr;          // cap
    // training buffers
    float *dh1 = nullptr, *dh2 = nullptr, *dra = nullptr, *drb = nullptr, *duh1 = nullptr, *da = nullptr;
    float* dgval = nullptr;          // cap * GW
    float* dgdiag = nullptr;         // cap
    float *z = nullptr, *v1 = nullptr, *v2 = nullptr;
    double* loss = nullptr;          // [4]: z^T M z, sum log G_ii
    float* dinv = nullptr;           // D^-1/2 per particle
    // The symmetric first-order form of G^T G on G's own pattern (both
    // triangles), S = G_d^2 + G_d G_L + G_L^T G_d (G_d the diagonal, G_L the
    // strict lower part), with the diagonal raised where needed so that S is
    // diagonally dominant and therefore SPD.  Kept by GEO index (particle id)
    // so that it stays valid across re-sorts between network evaluations.
    uint32_t* s_cnt = nullptr;       // cap: stored entries of the row (0: none, S_ii = 1)
    uint32_t* s_col = nullptr;       // cap * LP_GW: the neighbour's GEO index
    float* s_val = nullptr;          // cap * LP_GW: S_ij
    float* s_diag = nullptr;         // cap: S_ii
    bool s_ready = false;            // built at least once
};

int lp_setup(LearnedWork& L, uint32_t cap, std::string* err);
void lp_free(LearnedWork& L);
// default initial parameters (G = I: plain diagonal scaling) on the host
void lp_init_params(float* w, uint64_t seed);
void lp_upload_params(LearnedWork& L, const float* w, cudaStream_t st);

struct LpSystem {            // the assembled PPE system the network works on
    const float4* pos;       // positions at assembly (w = type bits)
    const float* n;          // particle number density
    const uint32_t* id;      // GEO.dat index (seeds the probe vectors)
    const uint32_t* rlen;    // PPE_DIRICHLET marks Dirichlet rows
    const double* diag64;    // diagonal of A (negative)
    const uint32_t* rowlist; // non-Dirichlet rows
    const uint32_t* nrows;
    const uint32_t* acols;   // rlap stencil, row-major stride PPE_W
    const uint32_t* cell;    // cell of each particle
    const uint32_t* cell_start;
    Grid g;
    Phys P;
    const Scalars* sc;
    // batch of scenes (null: one scene, g and P above): each row's scene
    // from its particle id, and that scene's grid (with its first global
    // cell) and constants
    const uint32_t* sid_of_id = nullptr;
    const Grid* grids = nullptr;
    const Phys* phys = nullptr;
};

// neighbours within r0 of every non-Dirichlet row, and D^-1/2
void lp_build_stencil(LearnedWork& L, const LpSystem& S, uint32_t cap, cudaStream_t st);
// network forward on the built stencil -> gdiag, gval (G and G^T values);
// tensor_cores: the 64 -> 64 layers on tcgen05 with BF16 activations, else
// in FP32 on the CUDA cores; keep_pre: store the pre-activations for the
// backward pass (the CUDA-core forward always does)
void lp_forward(LearnedWork& L, const LpSystem& S, bool exact, uint32_t cap, cudaStream_t st, bool tensor_cores,
                bool keep_pre = false);
// loss sums (L.loss = {z^T M z, sum log G_ii}) and the parameter gradient
// (L.grad) for a probe seed; the loss is lp_loss_value of those sums
int lp_loss_grad(LearnedWork& L, const LpSystem& S, bool exact, uint64_t seed, uint32_t cap, cudaStream_t st);
double lp_loss_value(const double* sums, uint32_t nrows);
// one Adam step on the FP32 master weights, then refresh the BF16 copy
void lp_adam(LearnedWork& L, float lr, cudaStream_t st);
// The symmetric form S by particle id (s_* arrays): allocate them, and
// build them after lp_forward (for np0 GEO indices)
int lp_alloc_symmetric(LearnedWork& L);
int lp_build_symmetric(LearnedWork& L, const LpSystem& S, uint32_t np0, cudaStream_t st);

}  // namespace mpsb
