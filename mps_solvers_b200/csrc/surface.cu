// surface.cu -- marching-cubes free surface (see surface.cuh).
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/mps_capi.h"
#include "cellsort.cuh"
#include "surface.cuh"

namespace mpsb {

static inline uint32_t blocks_for(uint32_t n, uint32_t t) { return (n + t - 1) / t; }

// ---------------------------------------------------------------- case table
static const int kCorner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                  {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
static const int kEdge[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                 {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
// the six faces as corner cycles
static const int kFace[6][4] = {{0, 1, 2, 3}, {4, 5, 6, 7}, {0, 1, 5, 4},
                                {1, 2, 6, 5}, {2, 3, 7, 6}, {3, 0, 4, 7}};

static int edge_of(int a, int b) {
    for (int e = 0; e < 12; e++)
        if ((kEdge[e][0] == a && kEdge[e][1] == b) || (kEdge[e][0] == b && kEdge[e][1] == a)) return e;
    return -1;
}

void mc_build_table(uint8_t ntri[256], int8_t tri[256][16]) {
    for (int c = 0; c < 256; c++) {
        memset(tri[c], -1, 16);
        ntri[c] = 0;
        auto in = [&](int k) { return (c >> k) & 1; };
        // segments: on each face, the crossing edges around each run of
        // inside corners
        int partner[12][2];
        int deg[12];
        for (int e = 0; e < 12; e++) deg[e] = 0;
        for (int f = 0; f < 6; f++) {
            const int* q = kFace[f];
            int nin = 0;
            for (int k = 0; k < 4; k++) nin += in(q[k]);
            if (nin == 0 || nin == 4) continue;
            for (int k = 0; k < 4; k++) {
                // a run starts at q[k] when q[k] is inside and its predecessor is not
                if (!in(q[k]) || in(q[(k + 3) % 4])) continue;
                int end = k;
                while (in(q[(end + 1) % 4])) end = (end + 1) % 4;
                const int ea = edge_of(q[(k + 3) % 4], q[k]);
                const int eb = edge_of(q[end], q[(end + 1) % 4]);
                partner[ea][deg[ea]++] = eb;
                partner[eb][deg[eb]++] = ea;
            }
        }
        // loops through the crossing edges (each has exactly two partners)
        bool used[12] = {false};
        int nt = 0;
        for (int e0 = 0; e0 < 12; e0++) {
            if (deg[e0] != 2 || used[e0]) continue;
            int loop[12], k = 0;
            int prev = -1, cur = e0;
            do {
                loop[k++] = cur;
                used[cur] = true;
                const int nxt = partner[cur][0] != prev ? partner[cur][0] : partner[cur][1];
                prev = cur;
                cur = nxt;
            } while (cur != e0 && k < 12);
            // orientation: loop normal (Newell, edge midpoints) along the
            // inside -> outside direction
            double mid[12][3], nrm[3] = {0, 0, 0}, out[3] = {0, 0, 0};
            for (int t = 0; t < k; t++) {
                const int a = kEdge[loop[t]][0], b = kEdge[loop[t]][1];
                const int ci = in(a) ? a : b, co = in(a) ? b : a;
                for (int d = 0; d < 3; d++) {
                    mid[t][d] = 0.5 * (kCorner[a][d] + kCorner[b][d]);
                    out[d] += kCorner[co][d] - kCorner[ci][d];
                }
            }
            for (int t = 0; t < k; t++) {
                const double* p = mid[t];
                const double* r = mid[(t + 1) % k];
                nrm[0] += (p[1] - r[1]) * (p[2] + r[2]);
                nrm[1] += (p[2] - r[2]) * (p[0] + r[0]);
                nrm[2] += (p[0] - r[0]) * (p[1] + r[1]);
            }
            if (nrm[0] * out[0] + nrm[1] * out[1] + nrm[2] * out[2] < 0) {
                for (int t = 0; t < k / 2; t++) {
                    const int s = loop[t];
                    loop[t] = loop[k - 1 - t];
                    loop[k - 1 - t] = s;
                }
            }
            for (int t = 1; t + 1 < k && nt < MC_MAX_TRI; t++) {
                tri[c][3 * nt] = (int8_t)loop[0];
                tri[c][3 * nt + 1] = (int8_t)loop[t];
                tri[c][3 * nt + 2] = (int8_t)loop[t + 1];
                nt++;
            }
        }
        ntri[c] = (uint8_t)nt;
    }
}

// ---------------------------------------------------------------- kernels
__device__ __forceinline__ float cubic_w(float r0, float r) {
    // MPS_GPU::r_cubic_weight (MPS_CAL_/MPS_GPU.cpp:54-62)
    const float q = r / r0;
    const float op = 0.31830988618379067f;  // 1/pi
    if (q <= 0.5f) return 8.0f * op * (1.f - 6.f * q * q + 6.f * q * q * q);
    if (q <= 1.0f) return 16.0f * op * (1.f - q) * (1.f - q) * (1.f - q);
    return 0.f;
}

// sum over the linked cells of w(r_ij; r0), j != i, every type; max over i
// (MPS_GPU::calOnce, MPS_CAL_/MPS_GPU.cpp:222-272)
__global__ void __launch_bounds__(256) k_surface_iso(StageArgs a, unsigned long long* best) {
    const uint32_t n = a.sc->np;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    float acc = 0.f;
    if (i < n) {
        const float4 pi = a.cur.pos[i];
        const Local L = local_of<false>(a, i);
        const int rows = link_rows(L.g);
        for (int row = 0; row < rows; row++) {
            const RowRange rg = link_row(L.g, L.cs, L.c, row);
            for (uint32_t j = rg.lo; j < rg.hi; j++) {
                if (j == i) continue;
                const float4 pj = __ldg(a.cur.pos + j);
                const float dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
                acc += cubic_w(a.P.rzero, sqrtf(dx * dx + dy * dy + dz * dz));
            }
        }
    }
    unsigned long long v = (unsigned long long)__float_as_uint(acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long t = __shfl_xor_sync(0xffffffffu, v, o);
        v = t > v ? t : v;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(best, v);
}

__global__ void k_surface_iso_set(const unsigned long long* best, uint32_t* out_bits) {
    out_bits[1] = __float_as_uint(0.8f * __uint_as_float((uint32_t)*best));
}

// vertex value: fluid particles within r0 of the vertex, from the cells
// that overlap [v - r0, v + r0], in ascending particle index
__global__ void __launch_bounds__(256) k_surface_vertex(StageArgs a, SurfaceGrid sg, float* __restrict__ vn) {
    const uint32_t nv = sg.nx * sg.ny * sg.nz;
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nv) return;
    const uint32_t ix = v % sg.nx, iy = (v / sg.nx) % sg.ny, iz = v / (sg.nx * sg.ny);
    const float x = sg.ox + sg.hx * ix, y = sg.oy + sg.hy * iy, z = sg.oz + sg.hz * iz;
    const Grid& g = a.g;
    const float r0 = a.P.rzero;
    auto cell_lo = [&](float p, float o, float h, uint32_t dim) {
        const float t = floorf((p - r0 - o) / h);
        return t < 0.f ? 0 : (t >= (float)dim ? (int)dim : (int)t);
    };
    auto cell_hi = [&](float p, float o, float h, uint32_t dim) {
        const float t = floorf((p + r0 - o) / h);
        return t < 0.f ? -1 : (t >= (float)dim ? (int)dim - 1 : (int)t);
    };
    const float hx = g.cell_size, hyz = g.cell_yz;
    const int x0 = cell_lo(x, g.left, hx, g.cdx), x1 = cell_hi(x, g.left, hx, g.cdx);
    const int y0 = cell_lo(y, g.back, hyz, g.cdy), y1 = cell_hi(y, g.back, hyz, g.cdy);
    const int z0 = g.dim == 3 ? cell_lo(z, g.bottom, hyz, g.cdz) : 0;
    const int z1 = g.dim == 3 ? cell_hi(z, g.bottom, hyz, g.cdz) : 0;
    float acc = 0.f;
    if (x0 <= x1) {
        for (int cz = z0; cz <= z1; cz++)
            for (int cy = y0; cy <= y1; cy++) {
                const uint32_t c0 = (uint32_t)cz * g.sheet + (uint32_t)cy * g.cdx;
                const uint32_t lo = __ldg(a.cell_start + c0 + (uint32_t)x0);
                const uint32_t hi = __ldg(a.cell_start + c0 + (uint32_t)x1 + 1u);
                for (uint32_t j = lo; j < hi; j++) {
                    const float4 pj = __ldg(a.cur.pos + j);
                    if (ptype(pj) != T_FLUID) continue;
                    const float dx = pj.x - x, dy = pj.y - y, dz = pj.z - z;
                    acc += cubic_w(r0, sqrtf(dx * dx + dy * dy + dz * dz));
                }
            }
    }
    vn[v] = acc;
}

__device__ __forceinline__ uint32_t cube_case(const float* __restrict__ vn, const SurfaceGrid& sg, uint32_t ix,
                                              uint32_t iy, uint32_t iz, float iso, float val[8]) {
    uint32_t idx = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const uint32_t cx = ix + (k == 1 || k == 2 || k == 5 || k == 6);
        const uint32_t cy = iy + (k == 2 || k == 3 || k == 6 || k == 7);
        const uint32_t cz = iz + (k >= 4);
        val[k] = vn[(cz * sg.ny + cy) * sg.nx + cx];
        idx |= (val[k] > iso ? 1u : 0u) << k;
    }
    return idx;
}

__global__ void __launch_bounds__(256) k_surface_count(const float* __restrict__ vn, SurfaceGrid sg,
                                                       const uint32_t* __restrict__ iso_bits,
                                                       const uint8_t* __restrict__ tab_n, uint32_t* __restrict__ cnt) {
    const uint32_t mx = sg.nx - 1, my = sg.ny - 1, mz = sg.nz - 1;
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c > mx * my * mz) return;
    if (c == mx * my * mz) {
        cnt[c] = 0;  // the scan's total slot
        return;
    }
    const float iso = __uint_as_float(iso_bits[1]);
    float val[8];
    const uint32_t idx = cube_case(vn, sg, c % mx, (c / mx) % my, c / (mx * my), iso, val);
    cnt[c] = tab_n[idx];
}

// -grad n at a vertex (central differences; one-sided at the grid's faces)
__device__ float3 vertex_normal(const float* __restrict__ vn, const SurfaceGrid& sg, uint32_t ix, uint32_t iy,
                                uint32_t iz) {
    auto at = [&](uint32_t x, uint32_t y, uint32_t z) { return vn[(z * sg.ny + y) * sg.nx + x]; };
    const uint32_t xm = ix > 0 ? ix - 1 : ix, xp = ix + 1 < sg.nx ? ix + 1 : ix;
    const uint32_t ym = iy > 0 ? iy - 1 : iy, yp = iy + 1 < sg.ny ? iy + 1 : iy;
    const uint32_t zm = iz > 0 ? iz - 1 : iz, zp = iz + 1 < sg.nz ? iz + 1 : iz;
    float3 g;
    g.x = (at(xp, iy, iz) - at(xm, iy, iz)) / (sg.hx * (float)(xp - xm > 0 ? xp - xm : 1));
    g.y = (at(ix, yp, iz) - at(ix, ym, iz)) / (sg.hy * (float)(yp - ym > 0 ? yp - ym : 1));
    g.z = (at(ix, iy, zp) - at(ix, iy, zm)) / (sg.hz * (float)(zp - zm > 0 ? zp - zm : 1));
    return make_float3(-g.x, -g.y, -g.z);
}

__global__ void __launch_bounds__(256) k_surface_emit(const float* __restrict__ vn, SurfaceGrid sg,
                                                      const uint32_t* __restrict__ iso_bits,
                                                      const uint8_t* __restrict__ tab_n, const int8_t* __restrict__ tab_t,
                                                      const uint32_t* __restrict__ off, uint32_t max_tri,
                                                      float* __restrict__ pos9, float* __restrict__ nrm9,
                                                      uint32_t* __restrict__ ntri) {
    const uint32_t mx = sg.nx - 1, my = sg.ny - 1, mz = sg.nz - 1;
    const uint32_t ncube = mx * my * mz;
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c == 0) ntri[0] = off[ncube];
    if (c >= ncube) return;
    const float iso = __uint_as_float(iso_bits[1]);
    const uint32_t ix = c % mx, iy = (c / mx) % my, iz = c / (mx * my);
    float val[8];
    const uint32_t idx = cube_case(vn, sg, ix, iy, iz, iso, val);
    const uint32_t nt = tab_n[idx];
    if (nt == 0) return;
    const uint32_t base = off[c];
    for (uint32_t t = 0; t < nt; t++) {
        if (base + t >= max_tri) return;
        for (int k = 0; k < 3; k++) {
            const int e = tab_t[idx * 16 + 3 * t + k];
            const int a = e < 4 ? e : (e < 8 ? e : e - 8);  // first corner of edge e
            int ca, cb;
            if (e < 4) { ca = e; cb = (e + 1) & 3; }
            else if (e < 8) { ca = e; cb = 4 + ((e - 4 + 1) & 3); }
            else { ca = a; cb = a + 4; }
            const float n1 = val[ca], n2 = val[cb];
            const float ax = sg.ox + sg.hx * (ix + (ca == 1 || ca == 2 || ca == 5 || ca == 6));
            const float ay = sg.oy + sg.hy * (iy + (ca == 2 || ca == 3 || ca == 6 || ca == 7));
            const float az = sg.oz + sg.hz * (iz + (ca >= 4));
            const float bx = sg.ox + sg.hx * (ix + (cb == 1 || cb == 2 || cb == 5 || cb == 6));
            const float by = sg.oy + sg.hy * (iy + (cb == 2 || cb == 3 || cb == 6 || cb == 7));
            const float bz = sg.oz + sg.hz * (iz + (cb >= 4));
            // the reference's vertexInterp (renderer_gpu_cudaker.cu:72-87)
            const float inv = 1.f / (n2 - n1);
            const size_t o = (size_t)(base + t) * 9 + 3 * k;
            pos9[o] = (iso * (bx - ax) + ax * n2 - bx * n1) * inv;
            pos9[o + 1] = (iso * (by - ay) + ay * n2 - by * n1) * inv;
            pos9[o + 2] = (iso * (bz - az) + az * n2 - bz * n1) * inv;
            const float s = (iso - n1) * inv;
            const float3 ga = vertex_normal(vn, sg, ix + (ca == 1 || ca == 2 || ca == 5 || ca == 6),
                                            iy + (ca == 2 || ca == 3 || ca == 6 || ca == 7), iz + (ca >= 4));
            const float3 gb = vertex_normal(vn, sg, ix + (cb == 1 || cb == 2 || cb == 5 || cb == 6),
                                            iy + (cb == 2 || cb == 3 || cb == 6 || cb == 7), iz + (cb >= 4));
            float nx = ga.x + s * (gb.x - ga.x), ny = ga.y + s * (gb.y - ga.y), nz = ga.z + s * (gb.z - ga.z);
            const float len = sqrtf(nx * nx + ny * ny + nz * nz);
            const float il = len > 0.f ? 1.f / len : 0.f;
            nrm9[o] = nx * il;
            nrm9[o + 1] = ny * il;
            nrm9[o + 2] = nz * il;
        }
    }
}

// ---------------------------------------------------------------- host
int surface_setup(SurfaceWork& w, const SurfaceGrid& g, uint32_t max_tri, cudaStream_t st, std::string* err) {
    surface_free(w);
    if (g.nx < 2 || g.ny < 2 || g.nz < 2 || !(g.hx > 0.f) || !(g.hy > 0.f) || !(g.hz > 0.f)) {
        *err = "surface grid needs at least 2 vertices and a positive spacing per axis";
        return MPS_ERR_INVALID;
    }
    const uint64_t nv = (uint64_t)g.nx * g.ny * g.nz;
    if (nv >= (1ull << 31)) {
        *err = "surface grid too large";
        return MPS_ERR_INVALID;
    }
    w.g = g;
    w.max_tri = max_tri;
    const uint64_t ncube = (uint64_t)(g.nx - 1) * (g.ny - 1) * (g.nz - 1);
    bool ok = true;
    auto al = [&](void** p, size_t bytes) {
        if (cudaMalloc(p, bytes + 64) != cudaSuccess) { ok = false; return; }
        cudaMemsetAsync(*p, 0, bytes + 64, st);
    };
    al((void**)&w.vn, nv * sizeof(float));
    al((void**)&w.cube_cnt, (ncube + 1) * sizeof(uint32_t));
    al((void**)&w.tri_pos, (size_t)max_tri * 9 * sizeof(float));
    al((void**)&w.tri_nrm, (size_t)max_tri * 9 * sizeof(float));
    al((void**)&w.ntri, 2 * sizeof(uint32_t));
    al((void**)&w.tab_n, 256);
    al((void**)&w.tab_t, 256 * 16);
    al((void**)&w.best, sizeof(unsigned long long));
    if (!ok) {
        *err = "cudaMalloc failed for the surface buffers";
        return MPS_ERR_CUDA;
    }
    uint8_t tn[256];
    int8_t tt[256][16];
    mc_build_table(tn, tt);
    cudaMemcpyAsync(w.tab_n, tn, 256, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(w.tab_t, tt, 256 * 16, cudaMemcpyHostToDevice, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        *err = "surface table upload failed";
        return MPS_ERR_CUDA;
    }
    w.ready = true;
    return MPS_OK;
}

void surface_enqueue_iso(SurfaceWork& w, const StageArgs& a, uint32_t cap, cudaStream_t st) {
    cudaMemsetAsync(w.best, 0, sizeof(unsigned long long), st);
    k_surface_iso<<<blocks_for(cap, 256), 256, 0, st>>>(a, w.best);
    k_surface_iso_set<<<1, 1, 0, st>>>(w.best, w.ntri);
}

void surface_enqueue_extract(SurfaceWork& w, const StageArgs& a, cudaStream_t st) {
    const SurfaceGrid& g = w.g;
    const uint32_t nv = g.nx * g.ny * g.nz;
    const uint32_t ncube = (g.nx - 1) * (g.ny - 1) * (g.nz - 1);
    k_surface_vertex<<<blocks_for(nv, 256), 256, 0, st>>>(a, g, w.vn);
    k_surface_count<<<blocks_for(ncube + 1, 256), 256, 0, st>>>(w.vn, g, w.ntri, w.tab_n, w.cube_cnt);
    launch_scan_exclusive(w.cube_cnt, ncube + 1, st);
    k_surface_emit<<<blocks_for(ncube, 256), 256, 0, st>>>(w.vn, g, w.ntri, w.tab_n, w.tab_t, w.cube_cnt, w.max_tri,
                                                           w.tri_pos, w.tri_nrm, w.ntri);
}

void surface_free(SurfaceWork& w) {
    void* ps[] = {w.vn, w.cube_cnt, w.tri_pos, w.tri_nrm, w.ntri, w.tab_n, w.tab_t, w.best};
    for (void* p : ps)
        if (p) cudaFree(p);
    w = SurfaceWork();
}

}  // namespace mpsb
