// mps_gpu_expl.hpp -- the reference's step-class interface on top of
// libmps_b200.so (include/mps_capi.h), header-only.
//
// A program written against the reference,
//
//     #include "MPS_GPU_EXPL.h"            // MPS_CAL_expl_v1.0/main.cpp:13-24
//     int main() { system("mkdir out");
//                  mytype::MPS_GPU_EXPL m; m.mps_cal(); return 0; }
//
// builds unchanged against this header (include it in place of
// MPS_GPU_EXPL.h) and links with -lmps_b200 -lcudart.  The class names,
// member names and their meaning follow MPS_CAL_expl_v1.0/MPS_GPU_EXPL.h:16-37
// (mps_cal, step) and MPS_CAL_/MPS_GPU.h:25,157-166 (Initial and the
// getters); MPS_CPU_EXPL (MPS_CAL_v4.0/MPS_CPU_EXPL.h:13-33) is the same
// class with the semi-implicit method.
//
// Differences a caller can see: getters return host copies refreshed after
// each step (the reference returns its own host arrays, also valid until
// the next step); errors end the process with the reference's exit codes
// (3 missing GEO.dat, 5 cells too thin, 1 dt too small, 4 particle outside
// the grid), and other library errors with exit code 7 after a message.
#pragma once
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "mps_capi.h"

namespace mytype {

struct real3 {
    float x, y, z;
};
typedef unsigned integer;

class MPS_GPU_EXPL {
public:
    explicit MPS_GPU_EXPL(int method = MPS_METHOD_EXPLICIT) : method_(method) {}
    ~MPS_GPU_EXPL() {
        if (h_) mps_destroy(h_);
    }
    MPS_GPU_EXPL(const MPS_GPU_EXPL&) = delete;
    MPS_GPU_EXPL& operator=(const MPS_GPU_EXPL&) = delete;

    // MPS_GPU::Initial: ./input.dat and ./GEO.dat of the working directory.
    void Initial() {
        mps_options o;
        mps_default_options(&o);
        o.method = method_;
        check(mps_create("input.dat", "GEO.dat", &o, &h_));
        stale_ = true;
    }
    // MPS_GPU_EXPL::step: one time step (plus i_step++, d_time += d_dt).
    void step() {
        if (!h_) Initial();
        check(mps_step(h_, 1, nullptr));
        stale_ = true;
    }
    // MPS_GPU_EXPL::mps_cal: initialise and run to tt with ./out/NNNN.out dumps.
    void mps_cal() {
        Initial();
        check(mps_run(h_, "./out"));
        stale_ = true;
    }

    const integer& getNp() const { refresh(); return np_; }
    const integer& getNb2() const { refresh(); return nb2_; }
    const integer& getNb1() const { refresh(); return nb1_; }
    integer* getId() const { refresh(); return id_.data(); }
    integer* getType() const { refresh(); return type_.data(); }
    real3* getPos() const { refresh(); return pos_.data(); }
    real3* getVel() const { refresh(); return vel_.data(); }
    float* getPres() const { refresh(); return press_.data(); }

protected:
    static int exit_code(mps_status s) {
        switch (s) {
            case MPS_ERR_IO: return 3;
            case MPS_ERR_CELLS_TOO_THIN: return 5;
            case MPS_ERR_DT_TOO_SMALL: return 1;
            case MPS_ERR_PARTICLE_OUT: return 4;
            default: return 7;
        }
    }
    void check(mps_status s) const {
        if (s == MPS_OK) return;
        std::fprintf(stderr, "mps: %s: %s\n", mps_status_string(s), h_ ? mps_last_error(h_) : "");
        std::exit(exit_code(s));
    }
    void refresh() const {
        if (!stale_ || !h_) return;
        uint32_t np = 0, nb2 = 0, nb1 = 0, nexcl = 0;
        check(mps_get_counts(h_, &np, &nb2, &nb1, &nexcl));
        np_ = np;
        nb2_ = nb2;
        nb1_ = nb1;
        id_.resize(np);
        type_.resize(np);
        pos_.resize(np);
        vel_.resize(np);
        press_.resize(np);
        check(mps_get_state(h_, id_.data(), type_.data(), reinterpret_cast<float*>(pos_.data()),
                            reinterpret_cast<float*>(vel_.data()), press_.data(), nullptr, MPS_ORDER_SORTED));
        stale_ = false;
    }

    int method_;
    mps_handle* h_ = nullptr;
    mutable bool stale_ = true;
    mutable integer np_ = 0, nb2_ = 0, nb1_ = 0;
    mutable std::vector<integer> id_, type_;
    mutable std::vector<real3> pos_, vel_;
    mutable std::vector<float> press_;
};

// The semi-implicit step class (MPS_CAL_v4.0/MPS_CPU_EXPL.h:13-33) on the GPU.
class MPS_CPU_EXPL : public MPS_GPU_EXPL {
public:
    MPS_CPU_EXPL() : MPS_GPU_EXPL(MPS_METHOD_SEMI_IMPLICIT) {}
};

// The GL build's step class (MPS_CAL_/MPS_GPU.h:18-166), driven as
//     mps = new mytype::MPS_GPU(); mps->Initial();   // MPS_CAL_/Renderer.h:54-56
//     ... mps->step(); ... mps->getPos() ...         // MPS_CAL_/Renderer.h:312
// Its step (MPS_CAL_/MPS_GPU.cpp:611-714) is the explicit equation-of-state
// step: viscosity, collision, PND, pressure, gradient, then update_dt and
// i_step++, the stages of MPS_GPU_EXPL::step.  Initial(), step() and the
// getters are inherited; the two public stage members run one stage:
class MPS_GPU : public MPS_GPU_EXPL {
public:
    MPS_GPU() : MPS_GPU_EXPL(MPS_METHOD_EXPLICIT) {}
    // MPS_GPU::calVisc_expl: viscosity and gravity on the fluid, applied to
    // velocities and positions (the library applies a stage's update while it
    // re-sorts the cells, so this runs the stage and then that rebuild).
    void calVisc_expl() {
        if (!h_) Initial();
        check(mps_phase(h_, 1));
        check(mps_phase(h_, 2));
        stale_ = true;
    }
    // MPS_GPU::calPres_expl: equation-of-state pressure from the current
    // number density, and the dummy particles' copy of their wall pressure.
    void calPres_expl() {
        if (!h_) Initial();
        check(mps_phase(h_, 5));
        stale_ = true;
    }
};

}  // namespace mytype
