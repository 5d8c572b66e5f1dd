/*
 * The drop-in boundary exercised from the reference's side: the maintainer's patch to
 * cJupiterModel::Run as a function over the reference's own model
 * object, compiled against the reference's headers where they lie and linked with the product's
 * C ABI library (atjup_b200/libatjup_gpu.so).
 *
 * TEST INFRASTRUCTURE: built by oracle/Makefile (target `dropin`) into oracle/_ref/, loaded only
 * by tests/test_dropin.py. It holds no hot-path code of its own: every step runs through
 * include/atjup_gpu.h.
 *
 * dropin_gpu_run(P, nm, solve) does, on the model ref_create built (the reference's
 * initialisation chain, cJupiterModel.cpp:316-760):
 *   - atjup_gpu_create with the caller's resolved AtjupParams,
 *   - atjup_gpu_set_grid from the model's rad, the, SeaMount, i_topography and cell-hold means,
 *   - atjup_gpu_upload_array of every field the dry iteration reads, from the model's jagged
 *     `double***` arrays (Array::x), and p_baro from its contiguous vector,
 *   - nm iterations of atjup_gpu_step (the loop of cJupiterModel.cpp:1010-1555),
 *   - atjup_gpu_download_array of the state back into the model's arrays, where the reference's
 *     own output writers and restart code would read it.
 */
// the standard headers the model's headers use, included before the access specifiers are
// opened (they must keep their own)
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <limits>
#include <map>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#define private public
#define protected public
#include "cJupiterModel.h"
#undef private
#undef protected

#include "atjup_gpu.h"

extern "C" void* ref_model_ptr(void);

namespace {

std::string g_err;

int fail(const char* what, int rc) {
    g_err = std::string(what) + ": " + atjup_gpu_last_error();
    return rc ? rc : 1;
}

}  // namespace

extern "C" {

const char* dropin_last_error(void) { return g_err.c_str(); }

int dropin_gpu_run(const AtjupParams* P, int32_t nm, const AtjupSolveOpts* solve) {
    cJupiterModel* mp = static_cast<cJupiterModel*>(ref_model_ptr());
    if (!mp || !P) { g_err = "no model (ref_create first) or no parameters"; return 1; }
    cJupiterModel& m = *mp;
    if (P->im != m.im || P->jm != m.jm || P->km != m.km) { g_err = "grid size mismatch"; return 1; }
    AtjupCtx* gpu = nullptr;
    int rc = atjup_gpu_create(P, &gpu);
    if (rc != ATJUP_OK) return fail("atjup_gpu_create", rc);
    // the static grid from the model's own arrays
    const int im = m.im, jm = m.jm, km = m.km;
    std::vector<uint8_t> solid((size_t)im * jm * km);
    std::vector<int32_t> topo((size_t)jm * km);
    for (int i = 0; i < im; i++)
        for (int j = 0; j < jm; j++)
            for (int k = 0; k < km; k++)
                solid[((size_t)i * jm + j) * km + k] = (m.SeaMount.x[i][j][k] == 1.0) ? 1 : 0;
    for (int j = 0; j < jm; j++)
        for (int k = 0; k < km; k++) topo[(size_t)j * km + k] = m.i_topography[j][k];
    const bool hold = !m.cell_vbar0.empty();
    rc = atjup_gpu_set_grid(gpu, m.rad.z, m.the.z, solid.data(), topo.data(),
                            hold ? m.cell_vbar0.data() : nullptr,
                            hold ? m.cell_ubar0.data() : nullptr);
    if (rc != ATJUP_OK) { atjup_gpu_destroy(gpu); return fail("atjup_gpu_set_grid", rc); }
    // the state the dry iteration reads, from the jagged arrays
    struct { int id; Array* a; } up[] = {
        {ATJUP_F_T, &m.t}, {ATJUP_F_U, &m.u}, {ATJUP_F_V, &m.v}, {ATJUP_F_W, &m.w},
        {ATJUP_F_P_DYN, &m.p_dyn}, {ATJUP_F_P_HYDRO, &m.p_hydro}, {ATJUP_F_P_STAT, &m.p_stat},
        {ATJUP_F_RHO_MIX, &m.rho_mix}, {ATJUP_F_WALL_NUE, &m.wall_nue},
        {ATJUP_F_AUX_U, &m.aux_u}, {ATJUP_F_AUX_V, &m.aux_v}, {ATJUP_F_AUX_W, &m.aux_w}};
    for (auto& f : up) {
        if ((rc = atjup_gpu_upload_array(gpu, f.id, f.a->x)) != ATJUP_OK) {
            atjup_gpu_destroy(gpu);
            return fail("atjup_gpu_upload_array", rc);
        }
    }
    if (!m.p_baro.empty() &&
        (rc = atjup_gpu_upload(gpu, ATJUP_F_P_BARO, m.p_baro.data())) != ATJUP_OK) {
        atjup_gpu_destroy(gpu);
        return fail("atjup_gpu_upload p_baro", rc);
    }
    // the loop
    for (int iter_n = 1; iter_n <= nm; iter_n++) {
        m.iter_n = iter_n;
        if ((rc = atjup_gpu_step(gpu, iter_n, iter_n == 1, solve)) != ATJUP_OK) {
            atjup_gpu_destroy(gpu);
            return fail("atjup_gpu_step", rc);
        }
    }
    // the state back into the model's arrays (the output cadence of the patch)
    struct { int id; Array* a; } down[] = {
        {ATJUP_F_T, &m.t}, {ATJUP_F_U, &m.u}, {ATJUP_F_V, &m.v}, {ATJUP_F_W, &m.w},
        {ATJUP_F_P_DYN, &m.p_dyn}, {ATJUP_F_P_HYDRO, &m.p_hydro}, {ATJUP_F_RHO_MIX, &m.rho_mix},
        {ATJUP_F_AUX_U, &m.aux_u}, {ATJUP_F_AUX_V, &m.aux_v}, {ATJUP_F_AUX_W, &m.aux_w}};
    for (auto& f : down) {
        if ((rc = atjup_gpu_download_array(gpu, f.id, f.a->x)) != ATJUP_OK) {
            atjup_gpu_destroy(gpu);
            return fail("atjup_gpu_download_array", rc);
        }
    }
    atjup_gpu_destroy(gpu);
    return 0;
}

}  // extern "C"
