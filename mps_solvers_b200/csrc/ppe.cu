// ppe.cu -- pressure Poisson equation of the semi-implicit step.
#include "ppe.cuh"

namespace mpsb {

int ppe_setup(PpeWork& w, uint32_t, const Grid&, const Phys&, const mps_params&, cudaStream_t, std::string* err) {
    w.ready = false;
    *err = "semi-implicit method not available in this build";
    return MPS_ERR_INVALID;
}
int ppe_enqueue(PpeWork&, const StageArgs&, const mps_options&, uint32_t, cudaStream_t) { return 0; }
void ppe_free(PpeWork& w) { w.ready = false; }

}  // namespace mpsb
