// ppe.cuh -- pressure Poisson equation of the semi-implicit step.
#pragma once
#include <cstdint>
#include <string>
#include <cuda_runtime.h>

#include "../../include/mps_capi.h"
#include "physics.cuh"

namespace mpsb {

struct PpeWork {
    bool ready = false;
};

int ppe_setup(PpeWork& w, uint32_t cap, const Grid& g, const Phys& P, const mps_params& prm, cudaStream_t st,
              std::string* err);
// returns the number of kernels enqueued
int ppe_enqueue(PpeWork& w, const StageArgs& a, const mps_options& opt, uint32_t cap, cudaStream_t st);
void ppe_free(PpeWork& w);

}  // namespace mpsb
