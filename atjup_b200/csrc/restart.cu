// Restart files of the device state in the reference's own format, so that a run can move between
// the CPU model and this library in either direction.
//
// Reference: cJupiterModel::save_state / load_state (FileIO_Jup.cpp:584-683) with the array lists
// restart_arrays() and restart_arrays_carried() (FileIO_Jup.cpp:281-304). The file is a header of
// five int32 (magic "JUP2" 0x4A555032, or "JUP1" 0x4A555031 without the carried arrays; im; jm;
// km; the iteration), then each array as im * jm rows of km doubles, then (JUP2) vel_star as jm
// rows of km doubles. The reference writes it after restoreVar, when every time-level-n copy
// equals its live field; the device keeps one copy of t, u, v, w and p_dyn (the state between
// steps is time level n), so tn, un, vn, wn and p_dynn are written from it, and the species and
// closure n copies from their own device copies. thermalmassflux, a diagnostic the device path
// does not compute (the step never reads it), is written as zeros. Reading skips the arrays the
// device does not hold and checks the magic, the grid and the file size before it touches the
// device.
//
// The reference's carried list is complete for its own runs, where the arrays below are zero or
// negligible, but the device's next iterations also read them when they are not: the NH4SH mass
// flux and the precipitation sinks of NH3 cloud and of the three CH4 species. carried = 2 appends
// them after vel_star in a marked trailer ("ATJX", a count, the arrays), which the reference's
// loader never reads (it stops after vel_star when its chromophore tracer is off), so that a file
// written here resumes bit-identically.
#include "ctx.cuh"

#include <algorithm>
#include <cstdio>
#include <sys/stat.h>

namespace atjup {
namespace {

enum Src { LIVE, NCOPY, ZERO };
struct Entry {
    int id;
    Src src;
};

// restart_arrays() in file order (FileIO_Jup.cpp:281-292)
const Entry kFixed[] = {
    {ATJUP_F_T, LIVE}, {ATJUP_F_U, LIVE}, {ATJUP_F_V, LIVE}, {ATJUP_F_W, LIVE},
    {ATJUP_F_T, LIVE}, {ATJUP_F_U, LIVE}, {ATJUP_F_V, LIVE}, {ATJUP_F_W, LIVE},   // tn .. wn
    {ATJUP_F_H2O, LIVE}, {ATJUP_F_H2O_CLOUD, LIVE}, {ATJUP_F_H2O_ICE, LIVE},
    {ATJUP_F_H2O, NCOPY}, {ATJUP_F_H2O_CLOUD, NCOPY}, {ATJUP_F_H2O_ICE, NCOPY},
    {ATJUP_F_H2S, LIVE}, {ATJUP_F_H2S, NCOPY},
    {ATJUP_F_NH3, LIVE}, {ATJUP_F_NH3_CLOUD, LIVE}, {ATJUP_F_NH3_ICE, LIVE},
    {ATJUP_F_NH3, NCOPY}, {ATJUP_F_NH3_CLOUD, NCOPY}, {ATJUP_F_NH3_ICE, NCOPY},
    {ATJUP_F_CH4, LIVE}, {ATJUP_F_CH4_CLOUD, LIVE}, {ATJUP_F_CH4_ICE, LIVE},
    {ATJUP_F_CH4, NCOPY}, {ATJUP_F_CH4_CLOUD, NCOPY}, {ATJUP_F_CH4_ICE, NCOPY},
    {ATJUP_F_NH4SH, LIVE}, {ATJUP_F_NH4SH, NCOPY},
    {ATJUP_F_P_DYN, LIVE}, {ATJUP_F_P_DYN, LIVE}, {ATJUP_F_P_STAT, LIVE},          // p_dyn, p_dynn
    {ATJUP_F_TKE, LIVE}, {ATJUP_F_DIS, LIVE}, {ATJUP_F_TKE, NCOPY}, {ATJUP_F_DIS, NCOPY},
    {ATJUP_F_NUE, LIVE},
};
// restart_arrays_carried() in file order (FileIO_Jup.cpp:298-304)
const Entry kCarried[] = {
    {ATJUP_F_AUX_U, LIVE}, {ATJUP_F_AUX_V, LIVE}, {ATJUP_F_AUX_W, LIVE},
    {ATJUP_F_DIFFLUX_H2S, LIVE}, {ATJUP_F_DIFFLUX_NH3, LIVE},
    {ATJUP_F_MASSFLUX_H2S, LIVE}, {ATJUP_F_MASSFLUX_NH3, LIVE},
    {ATJUP_F_FLUXLIM_NH4SH, LIVE}, {-1, ZERO},                                     // thermalmassflux
    {ATJUP_F_Q_PRECIP, LIVE}, {ATJUP_F_Q_RAD, LIVE}, {ATJUP_F_RHO_MIX, LIVE},
    {ATJUP_F_S_PRECIP_H2O, LIVE}, {ATJUP_F_S_PRECIP_H2O_CLOUD, LIVE},
    {ATJUP_F_S_PRECIP_H2O_ICE, LIVE}, {ATJUP_F_S_PRECIP_NH3, LIVE},
    {ATJUP_F_S_PRECIP_NH3_ICE, LIVE},
};
// the trailer of carried = 2
const Entry kExtra[] = {
    {ATJUP_F_MASSFLUX_NH4SH, LIVE}, {ATJUP_F_S_PRECIP_NH3_CLOUD, LIVE}, {ATJUP_F_S_PRECIP_CH4, LIVE},
    {ATJUP_F_S_PRECIP_CH4_CLOUD, LIVE}, {ATJUP_F_S_PRECIP_CH4_ICE, LIVE},
};
constexpr int kNExtra = (int)(sizeof(kExtra) / sizeof(kExtra[0]));
constexpr int32_t kExtraMagic = 0x41544A58;   // "ATJX"
constexpr int kNFixed = (int)(sizeof(kFixed) / sizeof(kFixed[0]));
constexpr int kNCarried = (int)(sizeof(kCarried) / sizeof(kCarried[0]));
constexpr int32_t kJup1 = 0x4A555031, kJup2 = 0x4A555032;

// the device buffer an entry reads from or writes to; nullptr for a zero array, or for an n copy
// when the physics block (which allocates the n copies) is not set: the live field stands in
const double* entry_ptr(const AtjupCtx* c, const Entry& e) {
    if (e.src == ZERO) return nullptr;
    if (e.src == NCOPY && c->fn[e.id]) return c->fn[e.id];
    return c->f[e.id];
}

struct File {
    FILE* f = nullptr;
    ~File() { if (f) fclose(f); }
};

}  // namespace
}  // namespace atjup

using namespace atjup;

extern "C" {

int atjup_gpu_save_state(AtjupCtx* c, const char* path, int32_t iter, int32_t carried) {
    if (!c || !path) { set_error("save_state: null argument"); return ATJUP_ERR_ARG; }
    const AtjupParams& P = c->P;
    File out;
    out.f = fopen(path, "wb");
    if (!out.f) { set_error(std::string("save_state: cannot open ") + path); return ATJUP_ERR_ARG; }
    const int32_t hdr[5] = {carried ? kJup2 : kJup1, P.im, P.jm, P.km, iter};
    const size_t rows = (size_t)P.im * P.jm, n = rows * P.km;
    std::vector<double> h(n);
    bool ok = fwrite(hdr, sizeof hdr, 1, out.f) == 1;
    auto put = [&](const Entry& e) -> int {
        const double* d = entry_ptr(c, e);
        if (!d) {
            std::fill(h.begin(), h.end(), 0.0);
        } else {
            ATJUP_CUDA(cudaMemcpy2DAsync(h.data(), sizeof(double) * P.km, d, sizeof(double) * c->KP,
                                         sizeof(double) * P.km, rows, cudaMemcpyDeviceToHost, c->stream));
            ATJUP_CUDA(cudaStreamSynchronize(c->stream));
        }
        ok = ok && fwrite(h.data(), sizeof(double), n, out.f) == n;
        return ATJUP_OK;
    };
    int rc = ATJUP_OK;
    for (int a = 0; a < kNFixed && rc == ATJUP_OK; a++) rc = put(kFixed[a]);
    if (carried) {
        for (int a = 0; a < kNCarried && rc == ATJUP_OK; a++) rc = put(kCarried[a]);
        if (rc == ATJUP_OK) {
            const size_t n2 = (size_t)P.jm * P.km;
            rc = [&]() -> int {
                ATJUP_CUDA(cudaMemcpy2DAsync(h.data(), sizeof(double) * P.km, c->f2[ATJUP_F2_VEL_STAR],
                                             sizeof(double) * c->KP, sizeof(double) * P.km, P.jm,
                                             cudaMemcpyDeviceToHost, c->stream));
                ATJUP_CUDA(cudaStreamSynchronize(c->stream));
                return ATJUP_OK;
            }();
            ok = ok && rc == ATJUP_OK && fwrite(h.data(), sizeof(double), n2, out.f) == n2;
        }
        if (carried == 2 && rc == ATJUP_OK) {
            const int32_t tr[2] = {kExtraMagic, kNExtra};
            ok = ok && fwrite(tr, sizeof tr, 1, out.f) == 1;
            for (int a = 0; a < kNExtra && rc == ATJUP_OK; a++) rc = put(kExtra[a]);
        }
    }
    if (rc != ATJUP_OK) return rc;
    if (!ok || fflush(out.f) != 0) {
        set_error(std::string("save_state: write failed (disk full?) for ") + path);
        return ATJUP_ERR_ARG;
    }
    return ATJUP_OK;
}

int atjup_gpu_load_state(AtjupCtx* c, const char* path, int32_t* iter, int32_t* carried) {
    if (!c || !path) { set_error("load_state: null argument"); return ATJUP_ERR_ARG; }
    const AtjupParams& P = c->P;
    File in;
    in.f = fopen(path, "rb");
    if (!in.f) { set_error(std::string("load_state: no file ") + path); return ATJUP_ERR_ARG; }
    int32_t hdr[5];
    if (fread(hdr, sizeof hdr, 1, in.f) != 1 || (hdr[0] != kJup1 && hdr[0] != kJup2) ||
        hdr[1] != P.im || hdr[2] != P.jm || hdr[3] != P.km) {
        set_error(std::string("load_state: bad header or grid mismatch in ") + path);
        return ATJUP_ERR_ARG;
    }
    const bool jup2 = hdr[0] == kJup2;
    const size_t rows = (size_t)P.im * P.jm, n = rows * P.km, n2 = (size_t)P.jm * P.km;
    const size_t need = sizeof hdr + sizeof(double) *
                        ((size_t)(kNFixed + (jup2 ? kNCarried : 0)) * n + (jup2 ? n2 : 0));
    struct stat st;
    if (fstat(fileno(in.f), &st) != 0 || (size_t)st.st_size < need) {
        set_error(std::string("load_state: truncated file ") + path);
        return ATJUP_ERR_ARG;
    }
    std::vector<double> h(n);
    auto get = [&](const Entry& e, bool dup) -> int {
        if (fread(h.data(), sizeof(double), n, in.f) != n) {
            set_error(std::string("load_state: read failed in ") + path);
            return ATJUP_ERR_ARG;
        }
        // duplicates (tn .. wn, p_dynn), the zero array and absent n copies are not held
        if (dup || e.src == ZERO || (e.src == NCOPY && !c->fn[e.id])) return ATJUP_OK;
        double* d = const_cast<double*>(entry_ptr(c, e));
        ATJUP_CUDA(cudaMemcpy2DAsync(d, sizeof(double) * c->KP, h.data(), sizeof(double) * P.km,
                                     sizeof(double) * P.km, rows, cudaMemcpyHostToDevice, c->stream));
        ATJUP_CUDA(cudaStreamSynchronize(c->stream));
        return ATJUP_OK;
    };
    int rc = ATJUP_OK;
    for (int a = 0; a < kNFixed && rc == ATJUP_OK; a++)
        rc = get(kFixed[a], (a >= 4 && a < 8) || a == 31);
    if (jup2) {
        for (int a = 0; a < kNCarried && rc == ATJUP_OK; a++) rc = get(kCarried[a], false);
        if (rc == ATJUP_OK) {
            if (fread(h.data(), sizeof(double), n2, in.f) != n2) {
                set_error(std::string("load_state: read failed in ") + path);
                return ATJUP_ERR_ARG;
            }
            ATJUP_CUDA(cudaMemcpy2DAsync(c->f2[ATJUP_F2_VEL_STAR], sizeof(double) * c->KP, h.data(),
                                         sizeof(double) * P.km, sizeof(double) * P.km, P.jm,
                                         cudaMemcpyHostToDevice, c->stream));
            ATJUP_CUDA(cudaStreamSynchronize(c->stream));
        }
    }
    // the trailer of carried = 2, when the file has one
    bool extra = false;
    if (jup2 && rc == ATJUP_OK && (size_t)st.st_size >= need + 2 * sizeof(int32_t) + sizeof(double) * kNExtra * n) {
        int32_t tr[2];
        if (fread(tr, sizeof tr, 1, in.f) == 1 && tr[0] == kExtraMagic && tr[1] == kNExtra) {
            for (int a = 0; a < kNExtra && rc == ATJUP_OK; a++) rc = get(kExtra[a], false);
            extra = true;
        }
    }
    if (rc != ATJUP_OK) return rc;
    if (iter) *iter = hdr[4];
    if (carried) *carried = jup2 ? (extra ? 2 : 1) : 0;
    return ATJUP_OK;
}

}  // extern "C"
