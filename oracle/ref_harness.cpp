// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY (never linked into the product).
//
// Drives the reference's own CPU step classes, compiled unmodified from the
// reference sources by oracle/Makefile (only the build switches in common.h
// are flipped: GPU_CUDA off, DIM, OMP_THREADS), and dumps their state in a
// small binary format that the tests and bench.py's CPU-baseline leg read.
//
//   REF_EXPL build: drives MPS_GPU_EXPL from MPS_CAL_expl_v1.0 (real = float),
//                   whose CPU `#else` branches are the explicit EOS step
//                   (MPS_CAL_expl_v1.0/MPS_GPU_EXPL.cpp:277-339).
//   REF_SEMI build: drives MPS_CPU_EXPL from MPS_CAL_v4.0 (real = double),
//                   the semi-implicit step with the dense PPE + CG
//                   (MPS_CAL_v4.0/MPS_CPU_EXPL.cpp:79-135).
//   REF_IMPL build: drives MPS_CPU_IMPL from MPS_CAL_v4.0, the same step with
//                   the viscosity by Crank-Nicolson (three dense CG solves)
//                   (MPS_CAL_v4.0/MPS_CPU_IMPL.cpp:79-338).
//
// usage: ref_{expl,semi,impl} <workdir> <nsteps> <dump_every> <out.bin> <threads>
//   workdir holds input.dat and GEO.dat (the reference reads both from the
//   current directory); stdout of the reference goes to workdir/stdout.txt.
//   Prints one JSON line on stderr with the step-loop wall time.
#include <cstdio>
#include <cstdlib>
#include <cstdint>
#include <cstring>
#include <ctime>
#include <unistd.h>
#include <fcntl.h>
#include <sys/stat.h>
#include <omp.h>

#ifdef REF_EXPL
#include "MPS_GPU_EXPL.h"
using namespace mytype;
typedef MPS_GPU_EXPL RefBase;
#elif defined(REF_IMPL)
#include "MPS_CPU_IMPL.h"
typedef MPS_CPU_IMPL RefBase;
#else
#include "MPS_CPU_EXPL.h"
typedef MPS_CPU_EXPL RefBase;
#endif

static void put_u32(FILE* f, uint32_t v) { fwrite(&v, 4, 1, f); }
static void put_f64(FILE* f, double v) { fwrite(&v, 8, 1, f); }

class Harness : public RefBase {
public:
    // mps_cal opens the log before Initial() (MPS_CAL_expl_v1.0/MPS_GPU_EXPL.cpp:222;
    // MPS_CAL_v4.0/MPS_CPU_EXPL.cpp:27); Initial() and the step write to it.
    void init() {
        fid_log = fopen("./out/LOG.txt", "at");
        Initial();
    }
    void finish() {
        if (fid_log) fclose(fid_log);
        fid_log = NULL;
    }
    void one_step() {
        // Same bookkeeping as the reference's mps_cal loop around step().
        step();
        i_step++;
        d_time += d_dt;
    }
    // Header: constants and the cell grid computed by the reference.
    void dump_header(FILE* f) {
        fwrite("MPSD", 1, 4, f);
        put_u32(f, 1);
        put_u32(f, (uint32_t)sizeof(real));
        put_u32(f, i_np);
        put_u32(f, i_nb2);
        put_u32(f, i_nb1);
        put_f64(f, d_nzero);
        put_f64(f, d_lambda);
        put_f64(f, d_cell_size);
        put_f64(f, d_cell_left);
        put_f64(f, d_cell_back);
        put_f64(f, d_cell_bottom);
        put_u32(f, i_cell_dx);
        put_u32(f, i_cell_dy);
        put_u32(f, i_cell_dz);
        put_u32(f, i_num_cells);
        // cell tables after the initial divideCell
        fwrite(i_cell_list, sizeof(integer), i_np, f);
        fwrite(i_cell_start, sizeof(integer), i_num_cells, f);
        fwrite(i_cell_end, sizeof(integer), i_num_cells, f);
#ifdef REF_EXPL
        fwrite(i_normal, sizeof(integer), i_np, f);
#else
        for (integer i = 0; i < i_np; i++) put_u32(f, 0xffffffffu);
#endif
    }
    void dump_state(FILE* f, uint32_t step_no) {
        put_u32(f, 0x53544550u);  // "STEP"
        put_u32(f, step_no);
        put_u32(f, i_np);
        put_f64(f, d_dt);
        put_f64(f, d_time);
        fwrite(i_id, sizeof(integer), i_np, f);
        fwrite(i_type, sizeof(integer), i_np, f);
        fwrite(d3_pos, sizeof(real3), i_np, f);
        fwrite(d3_vel, sizeof(real3), i_np, f);
        fwrite(d_press, sizeof(real), i_np, f);
        fwrite(d_n, sizeof(real), i_np, f);
    }
};

static double now_s() {
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

int main(int argc, char** argv) {
    if (argc < 6) {
        fprintf(stderr, "usage: %s workdir nsteps dump_every out.bin threads [untimed_first_steps]\n", argv[0]);
        return 2;
    }
    const char* workdir = argv[1];
    int nsteps = atoi(argv[2]);
    int dump_every = atoi(argv[3]);
    const char* out_path = argv[4];
    int threads = atoi(argv[5]);
    // the first `skip` steps run untimed, so that the timed steps are a
    // later window of the run (the one a GPU measurement times)
    int skip = argc > 6 ? atoi(argv[6]) : 0;

    // Resolve the output path before changing directory.
    char out_abs[4096];
    if (out_path[0] == '/') snprintf(out_abs, sizeof out_abs, "%s", out_path);
    else {
        char cwd[2048];
        if (!getcwd(cwd, sizeof cwd)) return 3;
        snprintf(out_abs, sizeof out_abs, "%s/%s", cwd, out_path);
    }
    if (chdir(workdir) != 0) { perror("chdir"); return 3; }
    mkdir("out", 0755);
    // The reference prints progress on stdout; keep it in a file.
    int fd = open("stdout.txt", O_WRONLY | O_CREAT | O_TRUNC, 0644);
    if (fd >= 0) { fflush(stdout); dup2(fd, 1); close(fd); }
    omp_set_num_threads(threads > 0 ? threads : 1);

    FILE* f = fopen(out_abs, "wb");
    if (!f) { perror("fopen out"); return 3; }

    Harness* h = new Harness();
    double t0 = now_s();
    h->init();
    double t_init = now_s() - t0;
    h->dump_header(f);
    h->dump_state(f, 0);
    double t_steps = 0.0;
    for (int s = 1; s <= nsteps; s++) {
        double a = now_s();
        h->one_step();
        if (s > skip) t_steps += now_s() - a;
        if (dump_every > 0 && (s % dump_every == 0 || s == nsteps)) h->dump_state(f, (uint32_t)s);
    }
    fclose(f);
    fflush(stdout);
    fprintf(stderr, "{\"init_s\": %.6f, \"steps\": %d, \"untimed_steps\": %d, \"steps_s\": %.6f, \"threads\": %d}\n",
            t_init, nsteps, skip < nsteps ? skip : nsteps, t_steps, threads);
    h->finish();
    delete h;
    return 0;
}
