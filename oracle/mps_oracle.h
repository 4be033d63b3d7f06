/* mps_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference's MPS step, used as the checker by tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg.  The product path
 * (libmps_b200.so) never links, loads or calls this code.
 *
 * Every function follows a reference function; the citations are given at
 * each definition in mps_oracle.c.  The restatement is written twice from one
 * template (mps_oracle_impl.inc): the *_f32 entry points evaluate in float
 * (the reference's `real` in MPS_CAL_expl_v1.0/typedef.h:72), the *_f64 ones
 * in double (MPS_CAL_v4.0/typedef.h:20).
 *
 * Pinning: tests/test_oracle_pin.py runs the reference binaries built by
 * oracle/Makefile (oracle/_ref/ref_expl, oracle/_ref/ref_semi) on the same
 * GEO.dat/input.dat and requires bit-identical state; the committed fixtures
 * under tests/golden/ were produced by that reference build.
 */
#ifndef MPS_ORACLE_H
#define MPS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* step variants */
enum {
    ORC_EXPL = 0,        /* MPS_GPU_EXPL::step, CPU branches (expl_v1.0)          */
    ORC_SEMI_SEQ = 1,    /* MPS_CPU_EXPL::step (v4.0) with its in-place loops run
                            sequentially in index order (one thread)           */
    ORC_SEMI_JACOBI = 2  /* v4.0 rules with every particle update two-phase
                            (read old state, then write): the race-free form
                            the GPU implements                                */
};

/* status codes (match include/mps_capi.h) */
enum {
    ORC_OK = 0, ORC_ERR_IO = 1, ORC_ERR_CELLS_TOO_THIN = 2, ORC_ERR_DT_TOO_SMALL = 3,
    ORC_ERR_PARTICLE_OUT = 4, ORC_ERR_CG_NOT_CONVERGED = 5
};

typedef struct orc_state orc_state;

/* f32 / f64 entry points share this signature set */
#define ORC_DECL(S, R)                                                                 \
    orc_state* orc_create_##S(const char* input_dat, const char* geo_dat, int variant,  \
                              int* status);                                            \
    void orc_destroy_##S(orc_state* st);                                               \
    int orc_step_##S(orc_state* st);                                                   \
    void orc_set_cg_##S(orc_state* st, int relative, double tol, int max_iter);        \
    void orc_set_body_force_##S(orc_state* st, double amp, double freq);               \
    int orc_add_wall_motion_##S(orc_state* st, const double* lo, const double* hi,      \
                                const double* vel, const double* amp, double freq,     \
                                double phase);                                         \
    void orc_clear_wall_motion_##S(orc_state* st);                                     \
    void orc_set_visc_implicit_##S(orc_state* st, int on);                             \
    void orc_counts_##S(const orc_state* st, uint32_t* np, uint32_t* nb2,              \
                        uint32_t* nb1, uint32_t* nexcl, uint32_t* ncells);             \
    void orc_scalars_##S(const orc_state* st, double* out16);                          \
    void orc_get_state_##S(const orc_state* st, uint32_t* id, uint32_t* type,          \
                           R* pos3, R* vel3, R* press, R* n);                          \
    void orc_set_state_##S(orc_state* st, const R* pos3, const R* vel3,                \
                           const R* press, const R* n);                                \
    void orc_get_cells_##S(const orc_state* st, uint32_t* cell_of, uint32_t* start,    \
                           uint32_t* end);                                             \
    void orc_get_normal_##S(const orc_state* st, uint32_t* normal);                    \
    int orc_divide_cell_##S(orc_state* st);                                            \
    int orc_cg_iters_##S(const orc_state* st);                                         \
    double orc_cg_relres_##S(const orc_state* st);                                     \
    void orc_phase_##S(orc_state* st, int phase);

ORC_DECL(f32, float)
ORC_DECL(f64, double)

#ifdef __cplusplus
}
#endif
#endif
