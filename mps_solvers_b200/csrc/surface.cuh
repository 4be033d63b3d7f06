// surface.cuh -- free-surface extraction by marching cubes (the reference's
// MPS_CAL_expl_gl_v3.1 iso-surface: MPS_GPU::calVertex_n, calTriangle and
// calNorm, gpu_kernel/renderer_gpu_cudaker.cu), as a headless triangle
// buffer instead of an OpenGL vertex buffer.
//
// Vertex value: n_v = sum over fluid particles j of the cubic spline
// w(|x_j - v|; r0) (8/pi (1 - 6q^2 + 6q^3) for q <= 1/2, 16/pi (1 - q)^3 for
// q <= 1, q = r/r0); iso = 0.8 * max over particles i of sum_{j != i}
// w(r_ij; r0) at set-up.  A cube corner is inside when n_v > iso.  Edge
// points interpolate linearly between the two corner values; normals are
// the normalised -grad n (central differences) interpolated the same way.
//
// The case table is generated here (mc_build_table), not copied: on each
// cube face the crossing edges are paired around every run of inside
// corners (inside corners of an ambiguous face are kept apart, a rule that
// only reads the face's four corners, so neighbouring cubes agree and the
// surface is closed); the segments link into loops, each loop is oriented
// with its normal pointing from inside to outside and fanned into
// triangles.  Corner and edge numbering: corners 0..3 the z = 0 face
// counter-clockwise from the origin, 4..7 above them; edges 0..3 and 4..7
// around those faces, 8..11 the vertical edges.
#pragma once
#include <cstdint>
#include <string>
#include <cuda_runtime.h>

#include "physics.cuh"

namespace mpsb {

constexpr int MC_MAX_TRI = 5;  // triangles a cube can hold

// ntri[case], tri[case][3 * t + k] = edge of vertex k of triangle t (-1 unused)
void mc_build_table(uint8_t ntri[256], int8_t tri[256][16]);

struct SurfaceGrid {
    uint32_t nx, ny, nz;       // vertices per axis
    float ox, oy, oz;          // first vertex
    float hx, hy, hz;          // spacing
};

struct SurfaceWork {
    bool ready = false;
    SurfaceGrid g{};
    float iso = 0.f;
    uint32_t max_tri = 0;
    float* vn = nullptr;          // vertex values
    uint32_t* cube_cnt = nullptr; // triangles per cube, then exclusive offsets
    float* tri_pos = nullptr;     // 9 floats per triangle
    float* tri_nrm = nullptr;     // 9 floats per triangle
    uint32_t* ntri = nullptr;     // [0] triangles found (may exceed max_tri), [1] iso bits
    uint8_t* tab_n = nullptr;     // 256
    int8_t* tab_t = nullptr;      // 256 * 16
    unsigned long long* best = nullptr;
};

int surface_setup(SurfaceWork& w, const SurfaceGrid& g, uint32_t max_tri, cudaStream_t st, std::string* err);
// iso = 0.8 * max_i sum_{j != i} w(r_ij; r0) over the current particles
void surface_enqueue_iso(SurfaceWork& w, const StageArgs& a, uint32_t cap, cudaStream_t st);
// vertex values, per-cube counts, offsets and the triangle buffer
void surface_enqueue_extract(SurfaceWork& w, const StageArgs& a, cudaStream_t st);
void surface_free(SurfaceWork& w);

}  // namespace mpsb
