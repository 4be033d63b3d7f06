// host_io.cpp -- reading the reference's input files and its text output.
// Compiled with -ffp-contract=off: every float expression here is evaluated
// as the reference evaluates it on x86-64 (one rounding per operation).
#include "host_io.h"

#include <cmath>
#include <cstdio>
#include <cstring>

namespace mpsb {

// MPS::loadCase (MPS_CAL_expl_v1.0/MPS.cpp:173-331): 16 pairs of lines, a
// label then a value; dim with %d, the rest with %f; r0, rlap and col_dis
// scaled by dp, dt_min by dt_max.
int read_input_dat(const char* path, mps_params* p, std::string* err) {
    FILE* f = fopen(path, "r");
    if (!f) {
        *err = std::string("cannot open ") + path;
        return MPS_ERR_IO;
    }
    char buf[256];
    float v[16] = {0};
    int dim = 0;
    for (int k = 0; k < 16; k++) {
        if (!fgets(buf, sizeof buf, f) || !fgets(buf, sizeof buf, f)) {
            fclose(f);
            *err = std::string("input.dat ended early: ") + path;
            return MPS_ERR_IO;
        }
        int ok = k == 0 ? sscanf(buf, "%d", &dim) : sscanf(buf, "%f", &v[k]);
        if (ok != 1) {
            fclose(f);
            *err = "input.dat: bad value for entry " + std::to_string(k);
            return MPS_ERR_IO;
        }
    }
    fclose(f);
    p->dim = dim;
    p->rho = v[1];
    p->niu = v[2];
    p->dp = v[3];
    p->rzero = v[4];
    p->rzero *= p->dp;
    p->rlap = v[5];
    p->rlap *= p->dp;
    p->beta = v[6];
    p->cs = v[7];
    p->cfl = v[8];
    p->col_dis = v[9];
    p->col_dis *= p->dp;
    p->col_rate = v[10];
    p->dt_max = v[11];
    p->dt_min = v[12];
    p->dt_min *= p->dt_max;
    p->tt = v[13];
    p->tout = v[14];
    p->max_dis = v[15];
    if (dim != 2 && dim != 3) {
        *err = "input.dat: dimension must be 2 or 3";
        return MPS_ERR_INVALID;
    }
    return MPS_OK;
}

// MPS::createGeo (MPS_CAL_expl_v1.0/MPS.cpp:336-407).
int read_geo_dat(const char* path, Geo* g, std::string* err) {
    FILE* f = fopen(path, "r");
    if (!f) {
        *err = std::string("no file '") + path + "' exist";
        return MPS_ERR_IO;
    }
    unsigned np = 0, nb2 = 0, nb1 = 0;
    if (fscanf(f, "%u %u %u", &np, &nb2, &nb1) != 3 || np == 0 || nb2 + nb1 > np) {
        fclose(f);
        *err = "GEO.dat: bad header";
        return MPS_ERR_IO;
    }
    g->np = np;
    g->nb2 = nb2;
    g->nb1 = nb1;
    g->pos.resize(3 * (size_t)np);
    g->vel.resize(3 * (size_t)np);
    g->press.resize(np);
    bool ok = true;
    for (unsigned i = 0; i < np && ok; i++) ok = fscanf(f, "%f%f%f", &g->pos[3 * i], &g->pos[3 * i + 1], &g->pos[3 * i + 2]) == 3;
    for (unsigned i = 0; i < np && ok; i++) ok = fscanf(f, "%f%f%f", &g->vel[3 * i], &g->vel[3 * i + 1], &g->vel[3 * i + 2]) == 3;
    for (unsigned i = 0; i < np && ok; i++) ok = fscanf(f, "%f", &g->press[i]) == 1;
    fclose(f);
    if (!ok) {
        *err = "GEO.dat: fewer values than np announces";
        return MPS_ERR_IO;
    }
    return MPS_OK;
}

// MPS::allocateCellList (MPS_CAL_expl_v1.0/MPS.cpp:567-619): bounding box of
// all particles widened by max_dis, cell = max(r0, rlap), at least 3 cells
// per axis.
int make_grid(const mps_params& p, const float* pos3, uint32_t np, HostGrid* out, std::string* err) {
    float cell_size = (p.rzero > p.rlap ? p.rzero : p.rlap);
    float left = pos3[0], right = pos3[0];
    float back = pos3[1], front = pos3[1];
    float bottom = pos3[2], top = pos3[2];
    for (uint32_t i = 0; i < np; i++) {
        const float* q = pos3 + 3 * (size_t)i;
        if (q[0] < left) left = q[0];
        if (q[0] > right) right = q[0];
        if (q[1] < back) back = q[1];
        if (q[1] > front) front = q[1];
        if (q[2] < bottom) bottom = q[2];
        if (q[2] > top) top = q[2];
    }
    left -= p.max_dis;
    right += p.max_dis;
    back -= p.max_dis;
    front += p.max_dis;
    bottom -= p.max_dis;
    top += p.max_dis;
    if (p.dim == 2) back = front = 0.0f;
    float dx = right - left, dy = front - back, dz = top - bottom;
    uint32_t cdx = (uint32_t)(dx / cell_size) + 1;
    uint32_t cdy = (uint32_t)(dy / cell_size) + 1;
    uint32_t cdz = (uint32_t)(dz / cell_size) + 1;
    if (cdx <= 2 || cdz <= 2 || (cdy <= 2 && p.dim == 3)) {
        char b[128];
        snprintf(b, sizeof b, "cells are too thin ! -> dx: %u, dy: %u, dz: %u", cdx, cdy, cdz);
        *err = b;
        return MPS_ERR_CELLS_TOO_THIN;
    }
    uint64_t ncells = (uint64_t)cdx * cdy * cdz;
    if (ncells >= 0x7fffffffull) {
        *err = "too many cells";
        return MPS_ERR_INVALID;
    }
    out->left = left;
    out->back = back;
    out->bottom = bottom;
    out->cell_size = cell_size;
    out->cdx = cdx;
    out->cdy = cdy;
    out->cdz = cdz;
    out->sheet = cdx * cdy;
    out->ncells = (uint32_t)ncells;
    out->dim = p.dim;
    out->cell_yz = cell_size;
    return MPS_OK;
}

bool refine_grid_yz(HostGrid* g) {
    if (g->dim != 3) return false;
    const uint64_t cdy = 2ull * g->cdy, cdz = 2ull * g->cdz;
    const uint64_t ncells = (uint64_t)g->cdx * cdy * cdz;
    if (ncells >= 0x7fffffffull) return false;
    g->cell_yz = 0.5f * g->cell_size;  // exact: same faces as the reference's cells, plus the midplanes
    g->cdy = (uint32_t)cdy;
    g->cdz = (uint32_t)cdz;
    g->sheet = g->cdx * g->cdy;
    g->ncells = (uint32_t)ncells;
    return true;
}

// MPS::calOnce constants (MPS_CAL_expl_v1.0/MPS.cpp:515-529) from n0, lambda.
void derive_constants(const mps_params& p, float nzero, float lambda_sum, HostConst* c) {
    c->nzero = nzero;
    c->lambda = lambda_sum / nzero;
    c->alpha = (float)(1.0 / (double)(p.rho * p.cs * p.cs));
    c->one_over_alpha = p.rho * p.cs * p.cs;
    c->one_over_rho = (float)(1.0 / (double)p.rho);
    c->one_over_nzero = (float)(1.0 / (double)c->nzero);
    c->one_over_dim = (float)(1.0 / (double)(float)p.dim);
    c->one_over_dt = (float)(1.0 / (double)p.dt_max);
    c->c_lap = (float)((2.0 * p.dim) / (double)(c->nzero * c->lambda));
}

// A float threshold T on r^2 such that every r^2 >= T has a correctly
// rounded square root strictly above r_edge (so the candidate fails both the
// reference's `r < re` and `ds <= col_dis` tests).
float rr_threshold(float r_edge) {
    float up = nextafterf(r_edge, INFINITY);
    double sq = (double)up * (double)up;
    float t = (float)sq;
    if ((double)t < sq) t = nextafterf(t, INFINITY);
    return t;
}

// MPS_GPU::writeCase (MPS_CAL_expl_v1.0/MPS_GPU.cpp:138-152) and
// MPS_CPU::writeCase (MPS_CAL_v4.0/MPS_CPU.cpp:127-140).
int write_case_text(const char* path, int format, uint32_t np, const uint32_t* id, const uint32_t* type,
                    const float* pos3, const float* vel3, const float* press) {
    FILE* f = fopen(path, "wt");
    if (!f) return MPS_ERR_IO;
    for (uint32_t i = 0; i < np; i++) {
        const float* x = pos3 + 3 * (size_t)i;
        const float* u = vel3 + 3 * (size_t)i;
        if (format == 0)
            fprintf(f, "%d %d %lf %lf %lf %lf %lf %lf %lf ", (int)id[i], (int)type[i], x[0], x[1], x[2], u[0], u[1],
                    u[2], press[i]);
        else
            fprintf(f, "%lf %lf %lf %lf %lf %lf %lf %d ", x[0], x[1], x[2], u[0], u[1], u[2], press[i], (int)id[i]);
    }
    fclose(f);
    return MPS_OK;
}

}  // namespace mpsb
