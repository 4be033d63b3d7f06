// host_io.h -- reference input files, grid set-up, constants, text output.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/mps_capi.h"

namespace mpsb {

struct Geo {
    uint32_t np = 0, nb2 = 0, nb1 = 0;
    std::vector<float> pos, vel, press;
};

struct HostGrid {
    float left, back, bottom, cell_size;
    uint32_t cdx, cdy, cdz, sheet, ncells;
    int dim;
    float cell_yz;  // cell edge along y and z: cell_size, or half of it on the refined grid
};

struct HostConst {
    float nzero, lambda, alpha, one_over_alpha, one_over_rho, one_over_nzero, one_over_dim, one_over_dt, c_lap;
};

int read_input_dat(const char* path, mps_params* p, std::string* err);
int read_geo_dat(const char* path, Geo* g, std::string* err);
int make_grid(const mps_params& p, const float* pos3, uint32_t np, HostGrid* out, std::string* err);
// The reference's grid with its cells halved along y and z (the fast-arithmetic
// 3-D path's grid); false, leaving the grid alone, for a 2-D grid or one whose
// refined cell count would not fit.
bool refine_grid_yz(HostGrid* g);
void derive_constants(const mps_params& p, float nzero, float lambda_sum, HostConst* c);
float rr_threshold(float r_edge);
int write_case_text(const char* path, int format, uint32_t np, const uint32_t* id, const uint32_t* type,
                    const float* pos3, const float* vel3, const float* press);

}  // namespace mpsb
