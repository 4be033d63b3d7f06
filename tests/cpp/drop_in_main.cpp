// A driver in the shape of the reference's main (create the output folder,
// construct the step class, run it), built against include/mps_gpu_expl.hpp.
#include <cstdlib>

#include "mps_gpu_expl.hpp"

int main() {
    if (std::system("mkdir -p out") != 0) return 2;
    mytype::MPS_GPU_EXPL mps;
    mps.mps_cal();
    return mps.getNp() > 0 ? 0 : 1;
}
