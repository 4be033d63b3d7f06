/* mps_capi.h -- C ABI of libmps_b200.so, the B200 (sm_100a) MPS particle step.
 *
 * This is the boundary a caller of the reference binds instead of the
 * reference's step classes.  The reference's interface is the C++ class chain
 * OBJECT -> MPS -> MPS_GPU -> MPS_GPU_EXPL (MPS_CAL_expl_v1.0/MPS_GPU_EXPL.h:16-37,
 * MPS_CAL_/MPS_GPU.h:18-166) and its CPU twin MPS_CPU_EXPL
 * (MPS_CAL_v4.0/MPS_CPU_EXPL.h:13-33); each entry point below names the member
 * it replaces.  include/mps_gpu_expl.hpp rebuilds that class interface on top
 * of these functions.
 *
 * Conventions: plain pointers and sizes only; every function returns an
 * mps_status (the reference calls exit(code) instead, see mps_status);
 * arrays passed in or out are HOST memory unless the name ends in _dev;
 * the library owns all device memory of a handle; one handle must be used
 * from one host thread at a time; every handle owns one CUDA stream.
 * Particle arrays are in the reference's cell-sorted order unless an
 * MPS_ORDER_BY_ID order is requested.
 */
#ifndef MPS_CAPI_H
#define MPS_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MPS_CAPI_VERSION 1

/* Status codes.  The reference's exit codes map as: exit(3) no GEO.dat
 * (MPS_CAL_expl_v1.0/MPS.cpp:340-345) -> MPS_ERR_IO; exit(5) cells too thin
 * (:610-619) -> MPS_ERR_CELLS_TOO_THIN; exit(1) dt below dt_min
 * (MPS_GPU.cpp:770-776) -> MPS_ERR_DT_TOO_SMALL; exit(4) particle outside the
 * grid (MPS_CAL_v4.0/MPS_CPU.cpp:172-176) -> MPS_ERR_PARTICLE_OUT (the
 * explicit method instead drops such particles as the reference's type 3 and
 * counts them, MPS_CAL_expl_v1.0/MPS_GPU.cpp:268-280). */
typedef enum {
    MPS_OK = 0,
    MPS_ERR_IO = 1,
    MPS_ERR_CELLS_TOO_THIN = 2,
    MPS_ERR_DT_TOO_SMALL = 3,
    MPS_ERR_PARTICLE_OUT = 4,
    MPS_ERR_CG_NOT_CONVERGED = 5,
    MPS_ERR_DEVICE_TIMEOUT = 6,
    MPS_ERR_CUDA = 7,
    MPS_ERR_NAN = 8,
    MPS_ERR_INVALID = 9,
    MPS_ERR_CAPACITY = 10
} mps_status;

/* Step methods. */
enum {
    /* MPS_GPU_EXPL::step: viscosity, collision, PND, equation-of-state
     * pressure, pressure gradient (MPS_CAL_expl_v1.0/MPS_GPU_EXPL.cpp:277-339). */
    MPS_METHOD_EXPLICIT = 0,
    /* MPS_CPU_EXPL::step: viscosity, collision, PND, pressure Poisson
     * equation solved by CG, clamp, gradient (MPS_CAL_v4.0/MPS_CPU_EXPL.cpp:79-135),
     * every particle update applied two-phase (old state read, then written). */
    MPS_METHOD_SEMI_IMPLICIT = 1
};

/* Arithmetic modes of the particle sums. */
enum {
    /* float operations in the reference's order with IEEE division and square
     * root and no fused multiply-add: the explicit step reproduces the
     * reference's float results bit for bit. */
    MPS_ARITH_EXACT = 0,
    /* fused multiply-add and a reciprocal-square-root weight; results agree
     * with MPS_ARITH_EXACT within float rounding. */
    MPS_ARITH_FAST = 1
};

/* PPE preconditioners (semi-implicit method). */
enum { MPS_PRECOND_DIAGONAL = 0, MPS_PRECOND_LEARNED = 1 };

/* Particle orders for getters. */
enum { MPS_ORDER_SORTED = 0, MPS_ORDER_BY_ID = 1 };

typedef struct {
    int method;          /* MPS_METHOD_*                                      */
    int arith;           /* MPS_ARITH_*                                       */
    int device;          /* CUDA device ordinal                               */
    int use_graph;       /* capture each step in a CUDA graph (1) or launch   */
    double cg_tol;       /* PPE: stop when |r| <= cg_tol * |b| (FP64 norms)   */
    int cg_max_iter;     /* PPE: iteration limit (0: 10000)                   */
    int cg_check_every;  /* PPE: most FP32 CG iterations between two FP64
                            true-residual checks (0: 1000)                   */
    int precond;         /* MPS_PRECOND_*                                     */
    uint32_t capacity;   /* particle capacity (0: the scene's np)             */
    int cg_inner_digits; /* PPE: the most decimal digits one FP32 inner solve
                            may reduce the residual by before the next FP64
                            check (0: 4)                                      */
    int ppe_pipelined;   /* PPE: 1 = pipelined single-reduction PCG (diagonal
                            scaling, single scenes); mps_autotune may change it */
    int ppe_l2_keep_mb;  /* PPE: MiB of the stored matrix read as evict_last so
                            it stays in L2 across CG iterations while the rest
                            streams as evict_first (0: half the L2; -1: no
                            hints)                                            */
    int visc_implicit;   /* semi-implicit single scenes: 1 = viscosity by
                            Crank-Nicolson, three PCG solves a step (the
                            reference's MPS_CPU_IMPL / MPS_GPU_IMPL step,
                            MPS_CAL_v4.0/MPS_CPU_IMPL.cpp:79-338); 0 = explicit */
    int rebuild_merge;   /* cell rebuilds: 0 = merge the particles that changed
                            cell into the sorted order when at most 8192
                            particles can move (fluid and moving walls), else
                            a full radix sort; -1 = always the full sort.  Both
                            give the same stable order.                       */
    int ppe_layout;      /* PPE matrix in the solver: 0 = compact (rows
                            numbered densely, 16-bit column codes, 6 bytes
                            per entry) for single scenes with diagonal
                            scaling, else the 8-byte layout; -1 = always the
                            8-byte layout.  Same matrix either way;
                            mps_autotune may change it.                       */
    int ppe_smem_chunks; /* 128-entry chunks of the matrix each warp keeps
                            in shared memory across CG iterations (0: 8;
                            -1: none; at most 8 in the compact layout, 6 in
                            the 8-byte layout with stored weights)           */
    int precond_every;   /* learned preconditioner (every layout, batches
                            too): steps between two evaluations of the
                            network; between them the symmetric form of the
                            factor is kept by particle (GEO index) and
                            re-packed for the current rows every step
                            (0: 40; 1: every step)                           */
} mps_options;

/* The 16 values of input.dat as the reference holds them after
 * MPS::loadCase: r0, rlap and col_dis already multiplied by dp, dt_min
 * already multiplied by dt_max (MPS_CAL_expl_v1.0/MPS.cpp:173-331). */
typedef struct {
    int dim;
    float rho, niu, dp, rzero, rlap, beta, cs, cfl, col_dis, col_rate, dt_max, dt_min, tt, tout,
        max_dis;
} mps_params;

typedef struct {
    uint32_t np;         /* active particles (the reference's i_np)            */
    uint32_t nexcl;      /* particles dropped for leaving the grid (i_nexcl)    */
    int step;            /* steps taken (i_step)                                */
    float time;          /* simulated time (d_time, float as in the reference)  */
    float dt;            /* dt of the last step (d_dt)                          */
    int cg_iters;        /* PPE iterations of the last step                     */
    double cg_relres;    /* final FP64 |b - Ax| / |b| of the last step          */
    int status;          /* sticky device error word mapped to mps_status      */
    float ms;            /* device time of the call (CUDA events on the stream) */
    uint32_t cg_outer;   /* FP64 true-residual passes of the last PPE solve    */
    uint32_t reserved[3];
} mps_step_stats;

typedef struct mps_handle mps_handle;

/* Grid of the reference's cell list (MPS::allocateCellList,
 * MPS_CAL_expl_v1.0/MPS.cpp:567-642).  cell_yz is the cell edge along y and
 * z; 0 (or cell_size) is the reference's cubic cell.  A handle created with
 * MPS_ARITH_FAST in 3-D sorts by the reference's grid with its cells halved
 * along y and z (cell_yz = cell_size / 2, cdy and cdz doubled), which its
 * stencil walks scan with fewer candidates; mps_get_grid and
 * mps_get_cell_tables report that grid.  Exact arithmetic keeps the
 * reference's grid. */
typedef struct {
    float left, back, bottom, cell_size;
    uint32_t cdx, cdy, cdz, ncells;
    int dim;
    float cell_yz;
} mps_grid;

const char* mps_status_string(mps_status s);
void mps_default_options(mps_options* opt);

/* MPS::loadCase + MPS::createGeo + MPS_GPU::Initial (MPS_CAL_expl_v1.0/MPS.cpp:173-407,
 * MPS_GPU.cpp:63-115): read input.dat and GEO.dat, build the cell grid, sort,
 * compute n0, lambda and the dummy-to-wall map on the device. */
mps_status mps_create(const char* input_dat, const char* geo_dat, const mps_options* opt,
                      mps_handle** out);
/* Same from memory: positions/velocities (3*np floats, x y z per particle),
 * pressures (np floats) in GEO.dat order (nb2 dummy, nb1 wall, then fluid). */
mps_status mps_create_from_arrays(const mps_params* p, uint32_t np, uint32_t nb2, uint32_t nb1,
                                  const float* pos3, const float* vel3, const float* press,
                                  const mps_options* opt, mps_handle** out);
void mps_destroy(mps_handle* h);

/* MPS_GPU_EXPL::step / MPS_CPU_EXPL::step, nsteps times, plus the mps_cal
 * loop's i_step++ and d_time += d_dt.  Asynchronous on the handle's stream
 * except that it waits for the steps to end to report stats (may be NULL). */
mps_status mps_step(mps_handle* h, int nsteps, mps_step_stats* stats);

/* Same steps, only enqueued on the handle's stream: returns without waiting
 * and reports no device error (the next mps_step, getter or
 * mps_step(h, 0, &stats) reports it). */
mps_status mps_step_async(mps_handle* h, int nsteps);

/* MPS_GPU_EXPL::mps_cal (MPS_CAL_expl_v1.0/MPS_GPU_EXPL.cpp:216-272): steps
 * while time < tt, writing out_dir/NNNN.out in the reference's text format
 * every tout (writeCase, MPS_GPU.cpp:138-152).  out_dir NULL: no output. */
mps_status mps_run(mps_handle* h, const char* out_dir);

/* getNp / getNb2 / getNb1 (MPS_CAL_/MPS_GPU.h:157-160). */
mps_status mps_get_counts(mps_handle* h, uint32_t* np, uint32_t* nb2, uint32_t* nb1,
                          uint32_t* nexcl);
/* getId / getType / getPos / getVel / getPres (MPS_CAL_/MPS_GPU.h:162-166) plus
 * the particle number density, copied into caller buffers of np (3*np)
 * entries; any pointer may be NULL.  order: MPS_ORDER_*; with BY_ID, entry k
 * is the particle whose GEO.dat index is k (np0 entries, dropped particles
 * get type 3 and zeros). */
mps_status mps_get_state(mps_handle* h, uint32_t* id, uint32_t* type, float* pos3, float* vel3,
                         float* press, float* n, int order);
/* Overwrite pos/vel/press/n of the active particles (sorted order); used to
 * drive single stages from a known state.  NULL pointers leave a field. */
mps_status mps_set_state(mps_handle* h, const float* pos3, const float* vel3, const float* press,
                         const float* n);
/* i_cell_list, i_cell_start, i_cell_end after the last divideCell
 * (MPS_CAL_expl_v1.0/MPS.h:41-45): np, ncells, ncells entries. */
mps_status mps_get_cell_tables(mps_handle* h, uint32_t* cell_of, uint32_t* start, uint32_t* end);
mps_status mps_get_grid(mps_handle* h, mps_grid* g);
/* n0, lambda, dt, time, c_lap = 2d/(n0 lambda), rho c^2, alpha, cg iterations,
 * cg relative residual, step, status, number of cells, kernels launched by
 * one step, FP64 residual passes of the last PPE solve, 1 when steps replay
 * a captured CUDA graph (0: direct launches), and the matrix entries of the
 * last PPE assembly whose column did not fit the compact layout's 16-bit
 * code (-1 when the solver uses the 8-byte layout). */
mps_status mps_get_scalars(mps_handle* h, double out16[16]);
/* i_normal as GEO.dat indices: for each particle (by GEO index) the GEO index
 * of its wall particle (itself when it has none), np0 entries. */
mps_status mps_get_normal_ids(mps_handle* h, uint32_t* normal_id);

/* One stage of the step (for per-stage parity tests):
 * 0 update_dt, 1 viscosity, 2 divideCell, 3 collision, 4 cal_n,
 * 5 EOS pressure + dummy copy, 6 pressure gradient + update, 7 PPE + clamp.
 * Stages 1, 3 and 6 leave their update pending; the next stage 2 applies it
 * while re-sorting, as the reference's divideCell follows each of them. */
mps_status mps_phase(mps_handle* h, int phase);

/* Per-stage device times: nsteps steps launched stage by stage (no graph)
 * with CUDA events between stages; stage_ms[k] (k < max_stages) receives the
 * summed milliseconds of stage k, *nstages the number of stages, and
 * mps_stage_name(k) its name (update_dt, visc, collision, pnd, pressure,
 * dash, step_end, cell_keys, radix_sort, cell_table, gather, ppe_solve,
 * motion; pressure is the dummy copy of the explicit method or the PPE
 * assembly of the semi-implicit one; radix_sort holds the cell keys and
 * their sort, by radix passes or, with the merge rebuild, the changed
 * particles' sort; cell_keys and cell_table are 0, their work done inside
 * radix_sort and gather).  The steps advance the simulation like mps_step. */
mps_status mps_profile_steps(mps_handle* h, int nsteps, double* stage_ms, int max_stages, int* nstages);
const char* mps_stage_name(int k);

/* ---- learned PPE preconditioner (no counterpart in the reference) --------
 * A factor G, lower triangular on each row's r0 neighbours, its entries
 * produced by a two-round message-passing network (hidden 64, GELU, BF16
 * weights, FP32 accumulation); the solvers apply M^-1 = D^-1/2 S D^-1/2 with
 * S the symmetric first-order form of G^T G on G's pattern, made diagonally
 * dominant (so SPD), re-evaluated every options.precond_every steps.
 * Selected with options.precond = MPS_PRECOND_LEARNED (semi-implicit
 * method).  The parameter vector has mps_precond_num_params() floats. */
uint32_t mps_precond_num_params(void);
mps_status mps_precond_get_params(mps_handle* h, float* w, uint32_t n);
/* Load parameters (also enables the network on a handle created with the
 * diagonal preconditioner, for training). */
mps_status mps_precond_set_params(mps_handle* h, const float* w, uint32_t n);
/* On the PPE system of the last step: the training loss
 * L = log(z^T M z / n) - (2/n) sum_i log G_ii, M = G Ahat G^T,
 * Ahat = D^-1/2 (-A) D^-1/2, n the number of unknowns and z a Rademacher
 * vector drawn from seed and the particle ids -- the logarithm of Kaporin's
 * condition number of M up to a constant of the system, with Hutchinson's
 * estimate of the trace -- and its gradient with respect to the FP32
 * parameters (n floats). */
mps_status mps_precond_loss_grad(mps_handle* h, uint64_t seed, double* loss, float* grad);
/* iters Adam steps (learning rate lr, probe seeds seed, seed+1, ...) on the
 * PPE system of the last step; loss of the first and last step. */
mps_status mps_precond_train(mps_handle* h, int iters, float lr, uint64_t seed, double* loss_first,
                             double* loss_last);
/* The state the last PPE system was assembled from (np entries each):
 * x y z type-bits per particle, n, GEO index, 1 for a solved (non-Dirichlet)
 * row, the diagonal of A. */
/* Run the network forward on the last PPE system with its 64 -> 64 layers
 * in FP32 on the CUDA cores and with BF16 activations on the tensor cores
 * (tcgen05, accumulators in tensor memory), report the largest difference
 * of the factor's entries relative to the largest entry, and keep the
 * tensor cores for inference when enable != 0 (training: the call below). */
mps_status mps_precond_tensor_cores(mps_handle* h, int enable, double* max_rel_diff);
/* Training (mps_precond_loss_grad, mps_precond_train) with the network's
 * 64 -> 64 layers on the tensor cores when enable != 0: the forward, the
 * input gradients dx = W^T dy and the weight gradients dW = sum dy x^T
 * (rows of the system as the contraction) with BF16 operands and FP32
 * accumulators in tensor memory.  0, the default, trains in FP32 on the CUDA
 * cores, the network the float64 oracle's gradients are checked against. */
mps_status mps_precond_train_tensor_cores(mps_handle* h, int enable);
mps_status mps_ppe_snapshot(mps_handle* h, float* pos4, float* n, uint32_t* id, uint32_t* is_row,
                            double* diag, uint32_t* count);
/* The off-diagonal entries of the last assembled PPE matrix exactly as the
 * solver stores them, i.e. the neighbour set of buildPoisson
 * (MPS_CAL_v4.0/MPS_CPU.cpp:651-698: j of type != 2 within rlap with a
 * nonzero weight and not a Dirichlet row) of each non-Dirichlet row i:
 * row_start (np + 1 entries, sorted particle order) and, when cols / weights
 * are not NULL, the columns (sorted particle indices, ascending) and their
 * weights in cols[row_start[i] .. row_start[i + 1]).  *nnz receives the
 * total; more than max_entries gives MPS_ERR_CAPACITY (call with cols =
 * weights = NULL first to size the buffers).  A debug getter like
 * mps_get_cell_tables; it allocates temporary device memory. */
mps_status mps_ppe_stencil(mps_handle* h, uint32_t* row_start, uint32_t* cols, float* weights,
                           uint64_t max_entries, uint64_t* nnz);

/* Bounded device waits.  The persistent PPE solvers synchronise their blocks
 * with grid-wide barriers; a barrier that is not complete after this many
 * nanoseconds of spinning sets MPS_ERR_DEVICE_TIMEOUT, every block returns,
 * and the next mps_step or getter reports the error (the context stays
 * usable).  0 restores the default of 1 s.  No counterpart in the reference,
 * which has no device-side waits (its host exit()s on errors,
 * MPS_CAL_/MPS_GPU.cpp:1449-1455); a very small limit makes the timeout path
 * testable without any fault. */
mps_status mps_set_device_wait_limit(mps_handle* h, uint64_t ns);

/* The handle's cudaStream_t, for callers that time or order work around it. */
mps_status mps_get_stream(mps_handle* h, void** stream);
/* Write the reference's text output for the current state:
 * format 0 = MPS_GPU::writeCase "id type x y z u v w p " (MPS_CAL_expl_v1.0/MPS_GPU.cpp:138-152),
 * format 1 = MPS_CPU::writeCase "x y z u v w p id " (MPS_CAL_v4.0/MPS_CPU.cpp:127-140). */
mps_status mps_write_case(mps_handle* h, const char* path, int format);
/* Text of the last error on this handle. */
const char* mps_last_error(mps_handle* h);

/* ---- device-pointer primitive: the neighbour-search rebuild ----------------
 * MPS_GPU::divideCell's ranking (MPS_CAL_expl_v1.0/MPS_GPU.cpp:248-315) on
 * device arrays: cell id of each of n particles (x y z w float4, w unused),
 * stable sort by cell, cell start/end tables.  perm_dev[new] = old index;
 * cell_of_dev[new] = cell id (ncells for a particle outside the grid, sorted
 * last); start_dev/end_dev get ncells entries; *n_in_grid_dev (device) the
 * count of particles inside the grid.  Scratch memory is allocated and freed
 * by the call; stream may be NULL (legacy default stream). */
mps_status mps_cell_sort_dev(const float* pos4_dev, uint32_t n, const mps_grid* g,
                             uint32_t* perm_dev, uint32_t* cell_of_dev, uint32_t* start_dev,
                             uint32_t* end_dev, uint32_t* n_in_grid_dev, void* stream);

/* ---- allocation-free variant of mps_cell_sort_dev -------------------------
 * No counterpart in the reference (the reference allocates and frees device
 * memory around every kernel call).  Same arguments, results and errors as
 * mps_cell_sort_dev, but it calls no cudaMalloc/cudaFree: its scratch is one
 * fixed device array of 10.25 MiB inside the library.  For callers that may
 * not allocate device memory themselves or through a library: hosts whose
 * pool allocator owns all device memory, and latency-critical loops where
 * the device-wide synchronisation of cudaMalloc/cudaFree is not acceptable.
 * Limits: n <= MPS_NOALLOC_MAX_PARTICLES and ncells <= MPS_NOALLOC_MAX_CELLS,
 * else MPS_ERR_CAPACITY.  All calls on a device share the array, so calls
 * whose GPU work overlaps race and must be serialised.  Every call looks the
 * array's address up for the current device and context (so it stays valid
 * after cudaDeviceReset).  The call waits for its stream before returning and
 * copies n from host memory, so it cannot be captured in a CUDA graph.  The
 * array stays allocated on every device that loaded the library until the
 * process exits. */
#define MPS_NOALLOC_MAX_PARTICLES 524288u
#define MPS_NOALLOC_MAX_CELLS 524288u
mps_status mps_cell_sort_dev_noalloc(const float* pos4_dev, uint32_t n, const mps_grid* g,
                                     uint32_t* perm_dev, uint32_t* cell_of_dev, uint32_t* start_dev,
                                     uint32_t* end_dev, uint32_t* n_in_grid_dev, void* stream);

/* ---- batches of scenes and the tank-acceleration body force ----
 * No counterpart in the reference, which runs one scene per process
 * (MPS_CAL_expl_v1.0/main.cpp:13-24).  A batch steps up to 256 scenes (each
 * its own input.dat / GEO.dat, grid, constants, dt and time) as one particle
 * set: every stage is one launch over all scenes, and the semi-implicit PPE
 * of all scenes is one persistent launch in which each scene runs its own
 * PCG to options.cg_tol (diagonally scaled, or with the learned form when
 * options.precond = MPS_PRECOND_LEARNED: mps_precond_set_params and
 * mps_precond_tensor_cores take batch handles; training takes single scenes).
 * Each scene evolves as it would in its own handle.
 * Particle ids of scene s are id_base(s) + its GEO.dat index;
 * mps_get_state(..., MPS_ORDER_BY_ID) returns all scenes in that order. */
typedef struct mps_scene_spec {
    const char* input_dat;
    const char* geo_dat;
    /* tank acceleration a(t) = accel_amp sin(2 pi accel_freq t) along x; the
     * viscosity stage's body force becomes g - a(t) (0: plain gravity) */
    float accel_amp;   /* m/s^2 */
    float accel_freq;  /* Hz */
    uint32_t reserved[4];
} mps_scene_spec;

typedef struct mps_scene_info {
    uint32_t id_base, np0, nb2, nb1;
    float time, dt, nzero, pad;
    int cg_iters, cg_outer;  /* the scene's last PPE solve */
    double cg_relres;
    uint32_t reserved[4];
} mps_scene_info;

mps_status mps_batch_create(const mps_scene_spec* scenes, uint32_t nscenes, const mps_options* opt,
                            mps_handle** out);
/* nsteps steps of every scene (the same as mps_step on a batch handle) */
mps_status mps_batch_step(mps_handle* h, int nsteps, mps_step_stats* stats);
mps_status mps_batch_scene_info(mps_handle* h, uint32_t scene, mps_scene_info* info);
/* Set the tank acceleration of a scene (scene 0 of a single-scene handle). */
mps_status mps_set_body_force(mps_handle* h, uint32_t scene, float accel_amp, float accel_freq);

/* ---- prescribed boundary motion ----
 * Replaces the reference's hook MOTION::doMotion(pos, vel, np)
 * (MPS_CAL_/MOTION.cpp:11-16), which MPS_GPU::motion (MPS_CAL_/MPS_GPU.cpp:
 * 1670-1673) calls as the first, commented-out statement of a step, before
 * divideCell (MPS_CAL_/MPS_GPU_EXPL.cpp:93-95).  mps_add_wall_motion selects
 * the wall and dummy particles (types 1 and 2) that lie inside [lo, hi] now
 * and belong to no earlier motion, and moves them rigidly from then on: at the
 * start of every step, with tau = time - (time of this call),
 *   x = x0 + vel tau + amp (sin(omega tau + phase) - sin(phase)),
 *   u = vel + amp omega cos(omega tau + phase),   omega = 2 pi freq,
 * x0 the position at selection, followed by a cell rebuild (a wave maker,
 * piston or oscillating plate).  Up to 8 motions per handle; single-scene
 * handles only.  *selected (may be NULL) receives the number of particles
 * taken.  The particles must stay inside the grid. */
mps_status mps_add_wall_motion(mps_handle* h, const float lo[3], const float hi[3], const float vel[3],
                               const float amp[3], float freq, float phase, uint32_t* selected);
/* Stop every motion; the moved particles stay where they are, at rest. */
mps_status mps_clear_wall_motion(mps_handle* h);

/* ---- free surface by marching cubes ----
 * The reference's iso-surface (MPS_CAL_expl_gl_v3.1: MPS_GPU::calVertex_n,
 * calTriangle, calNorm) as a headless triangle buffer.  Vertex value n_v =
 * sum over fluid particles of the cubic spline w(|x_j - v|; r0); iso = 0.8 x
 * the largest particle sum of w over its neighbours, taken at
 * mps_surface_setup (call it on the initial state to match the reference).
 * Triangles: 9 floats each (three vertices), normals likewise (the
 * normalised -grad n), counter-clockwise seen from the low-n side.
 * Single-scene handles only. */
typedef struct mps_surface_grid {
    uint32_t nx, ny, nz, pad;  /* vertices per axis */
    float origin[3];           /* first vertex */
    float spacing[3];
    uint32_t reserved[4];
} mps_surface_grid;
mps_status mps_surface_setup(mps_handle* h, const mps_surface_grid* grid, uint32_t max_triangles);
/* extract on the handle's stream (asynchronous) */
mps_status mps_surface_extract_async(mps_handle* h);
/* extract and wait; ntri = triangles found; MPS_ERR_CAPACITY when they
 * exceed max_triangles (the buffer then holds the first max_triangles) */
mps_status mps_surface_extract(mps_handle* h, uint32_t* ntri);
mps_status mps_surface_get(mps_handle* h, float* pos9, float* nrm9, uint32_t max_triangles, uint32_t* ntri);
/* vertex values (nx*ny*nz, x fastest) and the iso level */
mps_status mps_surface_vertex_values(mps_handle* h, float* values, float* iso);
/* the last extracted surface as a binary STL file */
mps_status mps_surface_write_stl(mps_handle* h, const char* path);
/* The marching-cubes case table the library generates (host only):
 * ntri[case] triangles, tri[16 * case + 3 * t + k] = cube edge of vertex k of
 * triangle t; bit k of case = corner k inside. */
mps_status mps_surface_case_table(uint8_t ntri[256], int8_t tri[256 * 16]);

/* ---- autotuner ----
 * No counterpart in the reference.  Times, on the handle's own scene with
 * CUDA events over `steps` steps per candidate, the block size of the
 * particle-stage kernels (64, 128, 256 threads) and, for the semi-implicit
 * PPE, the persistent grid's shape (1024, 512 or 256 threads per block at
 * 1024 threads per SM) and the solver's form (weights stored by the
 * assembly, weights recomputed from the positions in every product, or
 * stored weights with the pipelined single-reduction PCG, or the compact
 * 16-bit layout of options.ppe_layout), and keeps the fastest of each.
 * The scene advances by the steps taken (call it during warm-up). */
typedef struct mps_tune_report {
    int stage_threads;         /* chosen */
    int ppe_threads;           /* chosen */
    int ppe_stored_weights;    /* chosen: 1 stored, 0 recomputed */
    int ppe_pipelined;         /* chosen: 1 pipelined PCG */
    float stage_ms[3];         /* visc + collision + pnd + dash per step at 64, 128, 256 */
    /* PPE solve ms per step: [3 f + t] for form f (0 stored, 1 recomputed,
     * 2 pipelined) at 1024, 512, 256 threads per block (-1: not run) */
    float ppe_ms[9];
    int ppe_compact;           /* chosen: 1 the compact 16-bit layout        */
    float ppe_compact_ms[3];   /* its PPE solve ms per step at 1024, 512, 256
                                  threads per block (-1: not run)            */
} mps_tune_report;
mps_status mps_autotune(mps_handle* h, int steps, mps_tune_report* report);
/* Apply the choices of a report (the chosen fields: stage_threads,
 * ppe_threads, ppe_stored_weights, ppe_pipelined, ppe_compact) to a handle,
 * e.g. one tuned on a scratch handle of the same scene, without stepping. */
mps_status mps_apply_tuning(mps_handle* h, const mps_tune_report* report);

#ifdef __cplusplus
}
#endif
#endif
