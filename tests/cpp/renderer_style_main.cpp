// A driver in the shape of the reference GL build's use of its step class
// (MPS_CAL_/Renderer.h:54-56 and :312): construct MPS_GPU with new, call
// Initial(), then step() once per frame and read the particles through the
// raw getters, built against include/mps_gpu_expl.hpp.  Prints the particle
// count and sums of the state after the frames so the test can check it.
#include <cstdio>
#include <cstdlib>

#include "mps_gpu_expl.hpp"

int main(int argc, char** argv) {
    const int frames = argc > 1 ? std::atoi(argv[1]) : 10;
    mytype::MPS_GPU* mps = new mytype::MPS_GPU();
    mps->Initial();
    const mytype::integer np0 = mps->getNp();
    for (int f = 0; f < frames; f++) mps->step();
    const mytype::integer np = mps->getNp();
    const mytype::real3* pos = mps->getPos();
    const mytype::real3* vel = mps->getVel();
    const float* p = mps->getPres();
    const mytype::integer* type = mps->getType();
    double sz = 0.0, sw = 0.0, sp = 0.0;
    unsigned fluid = 0;
    for (mytype::integer i = 0; i < np; i++) {
        if (type[i] != 0) continue;
        fluid++;
        sz += pos[i].z;
        sw += vel[i].z;
        sp += p[i];
    }
    // one explicit stage pair through the public stage members
    mps->calVisc_expl();
    mps->calPres_expl();
    std::printf("%u %u %u %.9e %.9e %.9e %u\n", np0, np, fluid, sz, sw, sp, mps->getNp());
    delete mps;
    return np == np0 && fluid > 0 ? 0 : 1;
}
