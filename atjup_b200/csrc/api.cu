// C ABI of the B200 hot path: context, geometry, field transfer and the step schedule.
// The declarations and the reference routine each entry point replaces are in
// include/atjup_gpu.h.
#include "ctx.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

namespace atjup {

static thread_local std::string g_err;

void set_error(const std::string& msg) { g_err = msg; }

int cuda_status(cudaError_t e, const char* what) {
    g_err = std::string(what) + ": " + cudaGetErrorString(e);
    return ATJUP_ERR_CUDA;
}

int timer_begin(AtjupCtx* c, int cls, cudaStream_t st) {
    if (!c->timing) return -1;
    if ((size_t)(2 * c->tn + 2) > c->tev.size()) {
        for (int q = 0; q < 512; q++) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) { c->timing = false; return -1; }
            c->tev.push_back(e);
        }
    }
    const int n = c->tn++;
    c->tcls.resize(c->tn);
    c->tcls[n] = cls;
    cudaEventRecord(c->tev[2 * n], st);
    return n;
}

void timer_end(AtjupCtx* c, int slot, cudaStream_t st) {
    if (slot < 0) return;
    cudaEventRecord(c->tev[2 * slot + 1], st);
}

namespace {

// brackets the launches of one timing class with events on the compute stream (or on st)
struct Timed {
    AtjupCtx* c;
    cudaStream_t st;
    int slot;
    Timed(AtjupCtx* c_, int cls) : c(c_), st(c_->stream), slot(timer_begin(c_, cls, c_->stream)) {}
    Timed(AtjupCtx* c_, int cls, cudaStream_t s) : c(c_), st(s), slot(timer_begin(c_, cls, s)) {}
    ~Timed() { timer_end(c, slot, st); }
};

// The side stream: work that is independent of the compute stream's next launches runs on it
// (the scalar RK stages beside the dynamics stage, precipitation beside the closure update and
// the chemistry, the moist convective adjustment beside the velocity filters). fork_side orders
// the side stream after everything issued so far on the compute stream; join_side orders the
// compute stream after everything issued so far on the side stream.
int side_init(AtjupCtx* c) {
    if (c->side) return ATJUP_OK;
    ATJUP_CUDA(cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking));
    ATJUP_CUDA(cudaEventCreateWithFlags(&c->side_fork, cudaEventDisableTiming));
    ATJUP_CUDA(cudaEventCreateWithFlags(&c->side_join, cudaEventDisableTiming));
    return ATJUP_OK;
}
int fork_side(AtjupCtx* c) {
    if (int rc = side_init(c)) return rc;
    ATJUP_CUDA(cudaEventRecord(c->side_fork, c->stream));
    ATJUP_CUDA(cudaStreamWaitEvent(c->side, c->side_fork, 0));
    return ATJUP_OK;
}
int join_side(AtjupCtx* c) {
    ATJUP_CUDA(cudaEventRecord(c->side_join, c->side));
    ATJUP_CUDA(cudaStreamWaitEvent(c->stream, c->side_join, 0));
    return ATJUP_OK;
}
// issues the enclosed entry points on the side stream (they launch on c->stream)
struct OnSide {
    AtjupCtx* c;
    cudaStream_t main;
    explicit OnSide(AtjupCtx* c_) : c(c_), main(c_->stream) { c->stream = c->side; }
    ~OnSide() { c->stream = main; }
};

int alloc(double** p, size_t n) {
    ATJUP_CUDA(cudaMalloc(p, n * sizeof(double)));
    ATJUP_CUDA(cudaMemset(*p, 0, n * sizeof(double)));
    return ATJUP_OK;
}

void free_all(AtjupCtx* c) {
    xfer_free(c);
    if (c->side) {
        cudaStreamSynchronize(c->side);
        cudaEventDestroy(c->side_fork);
        cudaEventDestroy(c->side_join);
        cudaStreamDestroy(c->side);
        c->side = nullptr;
    }
    solver_free(c);
    cone_free(c);
    cudaFree(c->lin);
    c->lin = nullptr;
    cudaFree(c->itlin);
    c->itlin = nullptr;
    for (auto& p : c->f) { cudaFree(p); p = nullptr; }
    for (auto& p : c->f2) { cudaFree(p); p = nullptr; }
    for (auto& p : c->fn) { cudaFree(p); p = nullptr; }
    for (int q = 0; q < ATJUP_S_COUNT + 2; q++) {
        cudaFree(c->S1[q]); cudaFree(c->S2[q]); cudaFree(c->Sacc[q]);
        c->S1[q] = c->S2[q] = c->Sacc[q] = nullptr;
    }
    cudaFree(c->layer_h); c->layer_h = nullptr;
    cudaFree(c->cos_lat); c->cos_lat = nullptr;
    for (int q = 0; q < 4; q++) {
        cudaFree(c->X1[q]); cudaFree(c->X2[q]); cudaFree(c->acc[q]);
    }
    for (auto& p : c->kr) { cudaFree(p); p = nullptr; }
    for (auto& p : c->kf) { cudaFree(p); p = nullptr; }
    cudaFree(c->src); cudaFree(c->tmp); cudaFree(c->tmp2); cudaFree(c->red); cudaFree(c->stage);
    cudaFree(c->buoy_ref); cudaFree(c->zm); cudaFree(c->dvc); cudaFree(c->dvrow);
    cudaFree(c->mca_bounds); cudaFree(c->mca_flags); cudaFree(c->mca_slots); cudaFree(c->mca_stats);
    cudaFree(c->mca_pairs);
    cudaFree(c->solve_b); cudaFree(c->dsum); cudaFree(c->counters);
    if (c->hsum) cudaFreeHost(c->hsum);
    cudaFree(c->solid); cudaFree(c->nbflags); cudaFree(c->topo); cudaFree(c->geo); cudaFree(c->cor_col);
    cudaFree(c->sin_the); cudaFree(c->rad); cudaFree(c->cell_vbar0); cudaFree(c->cell_ubar0);
    cudaFree(c->solid_list); cudaFree(c->amb_rows); cudaFree(c->yw);
    cudaFree(c->line_a); cudaFree(c->line_c); cudaFree(c->line_m);
    for (auto e : c->tev) cudaEventDestroy(e);
    c->tev.clear();
}

bool valid_field(int id) { return id >= 0 && id < ATJUP_F_COUNT; }

// The Krylov/IR vectors are allocated on first use of the residual solver.
}  // namespace
}  // namespace atjup

using namespace atjup;

extern "C" {

void atjup_params_default(AtjupParams* p) {
    std::memset(p, 0, sizeof(*p));
    p->abi_version = ATJUP_ABI_VERSION;
    p->im = 41; p->jm = 181; p->km = 361;
    p->dr = 0.025;
    p->dthe = 1.0 / (180.0 / M_PI);
    p->dphi = 1.0 / (180.0 / M_PI);
    p->dt = 0.005;
    p->re = 1000.0; p->pr = 0.69; p->g = 25.92; p->omega = 0.000176; p->u_0 = 100.0;
    p->t_ref = 165.0; p->L_atm = 140.0;
    p->r_mix = 1.2843999999999998; p->R_mix = 3531.1847352206946; p->cp_mix = 11810.757033551794;
    p->Coriolis = 1.0; p->centrifugal = 1.0; p->buoyancy = 1.0;
    p->sinthe_min = 0.55;
    p->p_dyn_to_bar = p->r_mix * p->u_0 * p->u_0 * 1.0e-5;
    p->t_diff_scale = 0.01;
    p->nd_cor = p->L_atm * 1.0e3 / p->u_0;
    p->nd_cent = 1.0; p->nd_buoy = 1.0;
    p->buoy_scale = 1.0; p->buoy_ramp = 1.0; p->pgrad_scale = 1.0;
    p->rad_coupling = 1.0; p->precip_coupling = 1.0; p->turb_coupling = 1.0;
    p->pgrad_wall = 1; p->pgrad_wrap = 1; p->adiabatic = 1; p->adiabatic_rho = 1;
    p->metric_split = 1; p->coriolis_split = 1; p->hydro_split = 0; p->cell_hold = 1;
    p->precip_rho_local = 1; p->local_rho = 1; p->rho_pdyn = 0;
    p->has_nue = 0; p->has_heating = 0;
    p->p_dyn_cap = 0.2; p->press_wall = 1; p->rigid_lid = 1; p->press_sweeps = 1;
    p->top_taper = 3; p->lid_u = 1; p->pole_fill_rows = 2; p->mount_t_ambient = 1;
    p->shapiro_inloop = 0; p->shapiro_strength = 1.0;
    p->v_massbal_stride = 1; p->v_massbal_zonal = 1;
    p->precision = ATJUP_PREC_FP64;
    p->cone_proj_stride = 10; p->cone_proj_margin = 40; p->cone_proj_div = 3;
}

const char* atjup_gpu_last_error(void) { return g_err.c_str(); }

int atjup_gpu_create(const AtjupParams* params, AtjupCtx** out) {
    if (!params || !out) { set_error("create: null argument"); return ATJUP_ERR_ARG; }
    *out = nullptr;
    const AtjupParams& P = *params;
    if (P.abi_version != ATJUP_ABI_VERSION) { set_error("create: ABI version mismatch"); return ATJUP_ERR_ARG; }
    if (P.im < 5 || P.jm < 8 || P.km < 8 || ((P.km - 1) & 1)) {
        set_error("create: need im >= 5, jm >= 8, km >= 8 and an even number km-1 of meridians");
        return ATJUP_ERR_ARG;
    }
    if (!P.pgrad_wrap || !P.press_wall || !P.metric_split || P.hydro_split) {
        set_error("create: pgrad_wrap, press_wall and metric_split must be 1, hydro_split 0");
        return ATJUP_ERR_UNSUPPORTED;
    }
    if (P.top_taper < 0 || P.top_taper > 3 || P.pole_fill_rows < 0 || P.pole_fill_rows > 3) {
        set_error("create: top_taper must be 0..3, pole_fill_rows 0..3");
        return ATJUP_ERR_UNSUPPORTED;
    }
    if (P.cone_proj_stride < 0 || P.cone_proj_margin < 0 || P.cone_proj_div < 0) {
        set_error("create: cone_proj_stride, cone_proj_margin and cone_proj_div must be >= 0");
        return ATJUP_ERR_ARG;
    }
    if (P.precision != ATJUP_PREC_FP64 && P.precision != ATJUP_PREC_MIXED) {
        set_error("create: precision must be ATJUP_PREC_FP64 or ATJUP_PREC_MIXED");
        return ATJUP_ERR_ARG;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) { cuda_status(e, "cudaGetDevice"); return ATJUP_ERR_NO_DEVICE; }
    cudaDeviceProp prop;
    e = cudaGetDeviceProperties(&prop, dev);
    if (e != cudaSuccess) { cuda_status(e, "cudaGetDeviceProperties"); return ATJUP_ERR_NO_DEVICE; }
    if (prop.major != 10) {
        set_error("create: this library is built for sm_100a (B200); device is sm_" +
                  std::to_string(prop.major) + std::to_string(prop.minor));
        return ATJUP_ERR_NO_DEVICE;
    }
    AtjupCtx* c = new AtjupCtx();
    c->P = P;
    c->device = dev;
    c->step_prec = P.precision;
    c->KP = (P.km + 3 + 15) / 16 * 16;   // >= km + 3: 4-byte flag copies near the row end stay in the row
    c->NP = (size_t)P.im * P.jm * c->KP;
    int rc = ATJUP_OK;
    auto A = [&](double** p, size_t n) { if (rc == ATJUP_OK) rc = alloc(p, n); };
    for (int q = 0; q < ATJUP_F_COUNT; q++) A(&c->f[q], c->NP);
    for (int q = 0; q < ATJUP_F2_COUNT; q++) A(&c->f2[q], (size_t)P.jm * c->KP);
    for (int q = 0; q < 4; q++) { A(&c->X1[q], c->NP); A(&c->X2[q], c->NP); A(&c->acc[q], c->NP); }
    A(&c->src, c->NP);
    A(&c->tmp, c->NP);
    A(&c->tmp2, c->NP);
    A(&c->stage, (size_t)P.im * P.jm * P.km);
    A(&c->red, 4096);
    A(&c->buoy_ref, (size_t)P.im);
    A(&c->zm, (size_t)4 * P.jm);
    A(&c->dvc, (size_t)P.jm * c->KP);
    A(&c->dvrow, (size_t)P.jm);
    A(reinterpret_cast<double**>(&c->counters), 8);
    if (rc == ATJUP_OK) {
        e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) rc = cuda_status(e, "cudaStreamCreate");
        else c->own_stream = true;
    }
    if (rc != ATJUP_OK) { free_all(c); delete c; return rc; }
    *out = c;
    return ATJUP_OK;
}

int atjup_gpu_destroy(AtjupCtx* c) {
    if (!c) return ATJUP_OK;
    cudaStreamSynchronize(c->stream);
    free_all(c);
    if (c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
    return ATJUP_OK;
}

int atjup_gpu_set_stream(AtjupCtx* c, void* stream) {
    if (!c) return ATJUP_ERR_ARG;
    if (c->own_stream) { cudaStreamSynchronize(c->stream); cudaStreamDestroy(c->stream); }
    if (stream) { c->stream = (cudaStream_t)stream; c->own_stream = false; }
    else {
        ATJUP_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        c->own_stream = true;
    }
    return ATJUP_OK;
}

int atjup_gpu_copy_field(AtjupCtx* c, int32_t id, double* buf, int32_t to_field) {
    if (!c || !buf || !valid_field(id)) { set_error("copy_field: bad argument"); return ATJUP_ERR_ARG; }
    const size_t bytes = sizeof(double) * c->NP;
    if (to_field) ATJUP_CUDA(cudaMemcpyAsync(c->f[id], buf, bytes, cudaMemcpyDeviceToDevice, c->stream));
    else ATJUP_CUDA(cudaMemcpyAsync(buf, c->f[id], bytes, cudaMemcpyDeviceToDevice, c->stream));
    return ATJUP_OK;
}

int atjup_gpu_stream(AtjupCtx* c, void** stream) {
    if (!c || !stream) { set_error("stream: null argument"); return ATJUP_ERR_ARG; }
    *stream = (void*)c->stream;
    return ATJUP_OK;
}

int atjup_gpu_set_grid(AtjupCtx* c, const double* rad, const double* the, const uint8_t* solid,
                       const int32_t* i_topo, const double* cell_vbar0, const double* cell_ubar0) {
    if (!c || !rad || !the || !solid || !i_topo) { set_error("set_grid: null argument"); return ATJUP_ERR_ARG; }
    const AtjupParams& P = c->P;
    const int im = P.im, jm = P.jm, km = P.km, KP = c->KP;
    // geometry rows, built as RungeKutta_Jup_Turb.cpp:298-303, 388-411 builds them
    std::vector<GeoIJ> geo((size_t)im * jm);
    const double A = P.nd_cor * -2.0 * P.omega;
    for (int i = 0; i < im; i++)
        for (int j = 0; j < jm; j++) {
            GeoIJ& g = geo[(size_t)i * jm + j];
            std::memset(&g, 0, sizeof(g));
            const double rm = rad[i];
            const double rm2 = rm * rm;
            const double sinthe = std::max(P.sinthe_min, std::fabs(std::sin(the[j])));
            const double sinthe2 = sinthe * sinthe;
            const double costhe = std::cos(the[j]);
            g.rm = rm;
            g.inv_rm = 1.0 / rm;
            g.inv_rm2 = 1.0 / rm2;
            g.inv_rmsinthe = 1.0 / (rm * sinthe);
            g.inv_rm2sinthe = g.inv_rm2 / sinthe;
            g.inv_rm2sinthe2 = g.inv_rm2 / sinthe2;
            g.costhe_inv_rm2sinthe = costhe * g.inv_rm2sinthe;
            g.v_metric = (1.0 + costhe / (sinthe2)) * g.inv_rm2;
            g.cotanthe = costhe / sinthe;
            g.costhe = costhe;
            const double st = std::sqrt(std::max(0.0, 1.0 - costhe * costhe));
            g.sinthe_true = st;
            g.cent_rad = P.nd_cent * P.omega * P.omega * rm * st * st;
            g.cent_the = P.nd_cent * P.omega * P.omega * rm * st * costhe;
            g.cor_rad = A * st;
            g.cor_the = A * costhe;
            g.num2 = g.inv_rm2 * (1.0 / (P.dthe * P.dthe));
            g.num3 = g.inv_rm2sinthe2 * (1.0 / (P.dphi * P.dphi));
        }
    std::vector<double> cor_col(jm), sin_the(jm);
    for (int j = 0; j < jm; j++) {
        cor_col[j] = P.coriolis_split ? P.Coriolis * P.nd_cor * 2.0 * P.omega * std::fabs(std::sin(the[j])) : 0.0;
        sin_the[j] = std::sin(the[j]);
    }
    // padded mask
    std::vector<uint8_t> s_pad(c->NP, 0);
    for (size_t r = 0; r < (size_t)im * jm; r++)
        for (int k = 0; k < km; k++) s_pad[r * KP + k] = solid[r * km + k] ? 1 : 0;
    // per-cell flags for the RK stage: bit 0 solid, 1..6 solid neighbour (i+1, i-1, j+1, j-1,
    // k+1 and k-1 on the meridian ring), 7 integrated by the RK step
    std::vector<uint8_t> nbh(c->NP, 0);
    for (int i = 0; i < im; i++)
        for (int j = 0; j < jm; j++)
            for (int k = 0; k < km; k++) {
                auto S_ = [&](int ii, int jj, int kk) -> bool {
                    if (ii < 0 || ii >= im || jj < 0 || jj >= jm || kk < 0 || kk >= km) return false;
                    return solid[((size_t)ii * jm + jj) * km + kk] != 0;
                };
                const int ke = (k >= km - 2) ? 0 : k + 1, kw = (k == 0) ? km - 2 : k - 1;
                uint8_t f = 0;
                if (S_(i, j, k)) f |= 1;
                if (S_(i + 1, j, k)) f |= 2;
                if (S_(i - 1, j, k)) f |= 4;
                if (S_(i, j + 1, k)) f |= 8;
                if (S_(i, j - 1, k)) f |= 16;
                if (S_(i, j, ke)) f |= 32;
                if (S_(i, j, kw)) f |= 64;
                if (i >= 1 && i <= im - 2 && j >= 3 && j <= jm - 4 && k <= km - 2 && !(f & 1)) f |= 128;
                nbh[((size_t)i * jm + j) * KP + k] = f;
            }
    // solid-cell list for bcSolidGround (BC_Jup.h:496-590): first direction with two fluid cells
    auto sol = [&](int i, int j, int k) -> bool {
        if (i < 0 || i >= im || j < 0 || j >= jm || k < 0 || k >= km) return true;
        return solid[((size_t)i * jm + j) * km + k] != 0;
    };
    auto flu = [&](int i, int j, int k) -> bool {
        if (i < 0 || i >= im || j < 0 || j >= jm || k < 0 || k >= km) return false;
        return solid[((size_t)i * jm + j) * km + k] == 0;
    };
    std::vector<SolidCell> L;
    std::vector<int32_t> rows;
    for (int i = 0; i < im; i++)
        for (int j = 0; j < jm; j++) {
            bool any = false;
            for (int k = 0; k < km; k++) {
                if (!sol(i, j, k)) continue;
                any = true;
                SolidCell sc{};
                sc.c = (int64_t)(((size_t)i * jm + j) * KP + k);
                const bool surf = !sol(i + 1, j, k) || !sol(i - 1, j, k) || !sol(i, j + 1, k) ||
                                  !sol(i, j - 1, k) || !sol(i, j, k + 1) || !sol(i, j, k - 1);
                const int dirs[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
                sc.kind = 0;
                if (surf)
                    for (const auto& d : dirs)
                        if (flu(i + d[0], j + d[1], k + d[2]) && flu(i + 2 * d[0], j + 2 * d[1], k + 2 * d[2])) {
                            sc.kind = 1;
                            sc.a = (int64_t)(((size_t)(i + d[0]) * jm + (j + d[1])) * KP + (k + d[2]));
                            sc.b = (int64_t)(((size_t)(i + 2 * d[0]) * jm + (j + 2 * d[1])) * KP + (k + 2 * d[2]));
                            break;
                        }
                L.push_back(sc);
            }
            if (any) rows.push_back(i * jm + j);
        }
    if (!c->solid) {
        ATJUP_CUDA(cudaMalloc(&c->solid, c->NP));
        ATJUP_CUDA(cudaMalloc(&c->nbflags, c->NP));
        ATJUP_CUDA(cudaMalloc(&c->topo, sizeof(int32_t) * (size_t)jm * km));
        ATJUP_CUDA(cudaMalloc(&c->geo, sizeof(GeoIJ) * geo.size()));
        ATJUP_CUDA(cudaMalloc(&c->cor_col, sizeof(double) * jm));
        ATJUP_CUDA(cudaMalloc(&c->sin_the, sizeof(double) * jm));
        ATJUP_CUDA(cudaMalloc(&c->rad, sizeof(double) * im));
    }
    ATJUP_CUDA(cudaMemcpy(c->solid, s_pad.data(), c->NP, cudaMemcpyHostToDevice));
    ATJUP_CUDA(cudaMemcpy(c->nbflags, nbh.data(), c->NP, cudaMemcpyHostToDevice));
    ATJUP_CUDA(cudaMemcpy(c->topo, i_topo, sizeof(int32_t) * (size_t)jm * km, cudaMemcpyHostToDevice));
    ATJUP_CUDA(cudaMemcpy(c->geo, geo.data(), sizeof(GeoIJ) * geo.size(), cudaMemcpyHostToDevice));
    ATJUP_CUDA(cudaMemcpy(c->cor_col, cor_col.data(), sizeof(double) * jm, cudaMemcpyHostToDevice));
    ATJUP_CUDA(cudaMemcpy(c->sin_the, sin_the.data(), sizeof(double) * jm, cudaMemcpyHostToDevice));
    ATJUP_CUDA(cudaMemcpy(c->rad, rad, sizeof(double) * im, cudaMemcpyHostToDevice));
    cudaFree(c->cell_vbar0); cudaFree(c->cell_ubar0);
    c->cell_vbar0 = c->cell_ubar0 = nullptr;
    if (cell_vbar0 && cell_ubar0) {
        ATJUP_CUDA(cudaMalloc(&c->cell_vbar0, sizeof(double) * (size_t)im * jm));
        ATJUP_CUDA(cudaMalloc(&c->cell_ubar0, sizeof(double) * (size_t)im * jm));
        ATJUP_CUDA(cudaMemcpy(c->cell_vbar0, cell_vbar0, sizeof(double) * (size_t)im * jm, cudaMemcpyHostToDevice));
        ATJUP_CUDA(cudaMemcpy(c->cell_ubar0, cell_ubar0, sizeof(double) * (size_t)im * jm, cudaMemcpyHostToDevice));
    }
    cudaFree(c->solid_list); c->solid_list = nullptr;
    cudaFree(c->amb_rows); c->amb_rows = nullptr;
    c->n_solid = (int)L.size();
    c->n_amb_rows = (int)rows.size();
    if (c->n_solid > 0) {
        ATJUP_CUDA(cudaMalloc(&c->solid_list, sizeof(SolidCell) * L.size()));
        ATJUP_CUDA(cudaMemcpy(c->solid_list, L.data(), sizeof(SolidCell) * L.size(), cudaMemcpyHostToDevice));
        ATJUP_CUDA(cudaMalloc(&c->amb_rows, sizeof(int32_t) * rows.size()));
        ATJUP_CUDA(cudaMemcpy(c->amb_rows, rows.data(), sizeof(int32_t) * rows.size(), cudaMemcpyHostToDevice));
    }
    solver_free(c);                      // rebuilt by the residual solver for this mask
    cone_free(c);                        // and the projection's boxes
    c->grid_set = true;
    if (P.cone_proj_stride > 0) return cone_prepare(c);
    return ATJUP_OK;
}

// One contiguous host<->device copy through the staging buffer, and the row padding on the
// device (a pitched 2-D copy would move 7421 short rows per field).
int atjup_gpu_upload(AtjupCtx* c, int32_t id, const double* host) {
    if (!c || !host || !valid_field(id)) { set_error("upload: bad argument"); return ATJUP_ERR_ARG; }
    const AtjupParams& P = c->P;
    const size_t n = (size_t)P.im * P.jm * P.km;
    ATJUP_CUDA(cudaMemcpyAsync(c->stage, host, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
    int rc = launch_pad(c, c->stage, c->f[id]);
    if (rc) return rc;
    ATJUP_CUDA(cudaStreamSynchronize(c->stream));
    return ATJUP_OK;
}

int atjup_gpu_download(AtjupCtx* c, int32_t id, double* host) {
    if (!c || !host || !valid_field(id)) { set_error("download: bad argument"); return ATJUP_ERR_ARG; }
    const AtjupParams& P = c->P;
    const size_t n = (size_t)P.im * P.jm * P.km;
    int rc = launch_unpad(c, c->f[id], c->stage);
    if (rc) return rc;
    ATJUP_CUDA(cudaMemcpyAsync(host, c->stage, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
    ATJUP_CUDA(cudaStreamSynchronize(c->stream));
    return ATJUP_OK;
}

int atjup_gpu_upload_array(AtjupCtx* c, int32_t id, double*** x) {
    if (!c || !x || !valid_field(id)) { set_error("upload_array: bad argument"); return ATJUP_ERR_ARG; }
    const AtjupParams& P = c->P;
    std::vector<double> h((size_t)P.im * P.jm * P.km);
    for (int i = 0; i < P.im; i++)
        for (int j = 0; j < P.jm; j++)
            std::memcpy(&h[((size_t)i * P.jm + j) * P.km], x[i][j], sizeof(double) * P.km);
    return atjup_gpu_upload(c, id, h.data());
}

int atjup_gpu_download_array(AtjupCtx* c, int32_t id, double*** x) {
    if (!c || !x || !valid_field(id)) { set_error("download_array: bad argument"); return ATJUP_ERR_ARG; }
    const AtjupParams& P = c->P;
    std::vector<double> h((size_t)P.im * P.jm * P.km);
    int rc = atjup_gpu_download(c, id, h.data());
    if (rc != ATJUP_OK) return rc;
    for (int i = 0; i < P.im; i++)
        for (int j = 0; j < P.jm; j++)
            std::memcpy(x[i][j], &h[((size_t)i * P.jm + j) * P.km], sizeof(double) * P.km);
    return ATJUP_OK;
}

int atjup_gpu_field_ptr(AtjupCtx* c, int32_t id, void** dev_ptr, int32_t* pitch) {
    if (!c || !dev_ptr || !valid_field(id)) { set_error("field_ptr: bad argument"); return ATJUP_ERR_ARG; }
    *dev_ptr = c->f[id];
    if (pitch) *pitch = c->KP;
    return ATJUP_OK;
}

static int need_grid(AtjupCtx* c, const char* what) {
    if (!c) { set_error(std::string(what) + ": null context"); return ATJUP_ERR_ARG; }
    if (!c->grid_set) { set_error(std::string(what) + ": atjup_gpu_set_grid was not called"); return ATJUP_ERR_ARG; }
    return ATJUP_OK;
}

int atjup_gpu_set_stage_buffers(AtjupCtx* c, double* const bufs[12]) {
    if (!c) return ATJUP_ERR_ARG;
    if (!bufs) {
        c->keep_on = false;
        return ATJUP_OK;
    }
    for (int b = 0; b < 12; b++) {
        if (!bufs[b]) { set_error("set_stage_buffers: null buffer"); return ATJUP_ERR_ARG; }
        // the stage kernel reads its input through tensor maps, whose base must be 16-byte aligned
        if (reinterpret_cast<uintptr_t>(bufs[b]) % 16) {
            set_error("set_stage_buffers: buffers must be 16-byte aligned");
            return ATJUP_ERR_ARG;
        }
    }
    if (c->phys_on || c->step_prec != ATJUP_PREC_FP64) {
        set_error("set_stage_buffers: the FP64 dry step only");
        return ATJUP_ERR_UNSUPPORTED;
    }
    for (int b = 0; b < 12; b++) c->keep[b] = bufs[b];
    c->keep_on = true;
    return ATJUP_OK;
}

int atjup_gpu_rk4_step(AtjupCtx* c, int32_t iter_n) {
    (void)iter_n;
    int rc = need_grid(c, "rk4_step");
    if (rc) return rc;
    double* Y[4] = {c->f[ATJUP_F_T], c->f[ATJUP_F_U], c->f[ATJUP_F_V], c->f[ATJUP_F_W]};
    {
        Timed tm(c, TK_RK_AUX);
        if ((rc = launch_buoy_ref(c, Y[0]))) return rc;
        if ((rc = launch_hydrostatic(c, Y[2], Y[3]))) return rc;
    }
    // stage buffers: doubles, or in the mixed step floats in the first half of each buffer
    const void* in0[4] = {Y[0], Y[1], Y[2], Y[3]};
    const void* in1[4] = {c->X1[0], c->X1[1], c->X1[2], c->X1[3]};
    const void* in2[4] = {c->X2[0], c->X2[1], c->X2[2], c->X2[3]};
    void* out1[4] = {c->X1[0], c->X1[1], c->X1[2], c->X1[3]};
    void* out2[4] = {c->X2[0], c->X2[1], c->X2[2], c->X2[3]};
    const void* const* ins[4] = {in0, in1, in2, in1};
    void* const* outs[4] = {out1, out2, out1, nullptr};
    // the caller's stage buffers (atjup_gpu_set_stage_buffers): X1, X2, X3 each kept
    const void* kin[3][4];
    void* kout[3][4];
    if (c->keep_on && !c->phys_on && c->step_prec == ATJUP_PREC_FP64) {
        for (int s = 0; s < 3; s++)
            for (int f = 0; f < 4; f++) kin[s][f] = kout[s][f] = c->keep[4 * s + f];
        for (int f = 0; f < 4; f++) in1[f] = kin[0][f];
        ins[1] = kin[0]; ins[2] = kin[1]; ins[3] = kin[2];
        outs[0] = kout[0]; outs[1] = kout[1]; outs[2] = kout[2];
    }
    // The species and closure kernels of stage s read the stage input ins[s] and write only scalar
    // buffers; the dynamics kernel of stage s reads ins[s] too and writes outs[s], which is the
    // input the scalars of stage s - 1 read (X1 for stage 2, the FP64 state for stage 3). So the
    // scalars of stage s run on the side stream beside the dynamics of stage s: they start after
    // the dynamics of stage s - 1 (fork), and the dynamics of stage s + 1 starts after them (join).
    const bool fork = c->phys_on && (c->phys.species_on || c->phys.turb_on);
    for (int s = 0; s < 4; s++) {
        // timing slots of the stage: the dynamics kernel's, the side stream's first and last (the
        // stage's span is read from them; an event of its own here would change how the two
        // streams' kernels share the GPU)
        int side_first = -1, side_last = -1, dyn = -1;
        if (fork) {
            if ((rc = fork_side(c))) return rc;
            if (c->phys.species_on) {
                Timed tm(c, TK_SPECIES, c->side);
                side_first = side_last = tm.slot;
                if ((rc = launch_phys_stage(c, s, ins[s], 0, c->side))) return rc;
            }
            if (c->phys.turb_on) {
                Timed tm(c, TK_CLOSURE, c->side);
                if (side_first < 0) side_first = tm.slot;
                side_last = tm.slot;
                if ((rc = launch_phys_stage(c, s, ins[s], 1, c->side))) return rc;
            }
        }
        {
            Timed tm(c, TK_RK_STAGE);
            dyn = tm.slot;
            if ((rc = launch_rk_stage(c, s, ins[s], outs[s], in1))) return rc;
        }
        if (fork && (rc = join_side(c))) return rc;
        if (dyn >= 0) {
            c->tgrp.push_back(dyn);
            c->tgrp.push_back(side_first);
            c->tgrp.push_back(side_last);
        }
    }
    return ATJUP_OK;
}

int atjup_gpu_set_precision(AtjupCtx* c, int32_t prec) {
    if (!c) { set_error("set_precision: null context"); return ATJUP_ERR_ARG; }
    if (prec != ATJUP_PREC_FP64 && prec != ATJUP_PREC_MIXED) {
        set_error("set_precision: precision must be ATJUP_PREC_FP64 or ATJUP_PREC_MIXED");
        return ATJUP_ERR_ARG;
    }
    c->step_prec = prec;      // every stage buffer is rewritten by the next step's stage 0
    c->P.precision = prec;
    return ATJUP_OK;
}

int atjup_gpu_set_mca(AtjupCtx* c, const AtjupMca* m) {
    if (!c) { set_error("set_mca: null context"); return ATJUP_ERR_ARG; }
    if (!m) { c->mca_on = false; return ATJUP_OK; }
    if (!c->micro_on || !c->phys_on || !c->layer_h) {
        set_error("set_mca: needs atjup_gpu_set_physics and atjup_gpu_set_micro first");
        return ATJUP_ERR_ARG;
    }
    c->mca = *m;
    c->mca_on = m->stride > 0;
    return mca_setup(c);
}

int atjup_gpu_mca(AtjupCtx* c, AtjupMcaStats* st) {
    if (!c || !c->mca_bounds || !c->micro_on) { set_error("mca: atjup_gpu_set_mca was not called"); return ATJUP_ERR_ARG; }
    {
        Timed tm(c, TK_MCA);
        int rc = launch_mca(c);
        if (rc) return rc;
    }
    if (st) {
        unsigned long long h[8];
        int rc = mca_read_stats(c, h);
        if (rc) return rc;
        st->columns = (int64_t)h[0]; st->layers = (int64_t)h[1];
        st->moist_triggers = (int64_t)h[2]; st->dry_triggers = (int64_t)h[3];
        st->unstable_t = (int64_t)h[4]; st->held = (int64_t)h[5]; st->skipped = (int64_t)h[6];
        st->max_passes = (int32_t)h[7]; st->pad = 0;
    }
    return ATJUP_OK;
}

int atjup_gpu_set_physics(AtjupCtx* c, const AtjupPhysics* ph, const float* layer_heights_km) {
    if (!c) { set_error("set_physics: null context"); return ATJUP_ERR_ARG; }
    if (!ph) { c->phys_on = false; return ATJUP_OK; }
    if (!layer_heights_km) { set_error("set_physics: layer heights required"); return ATJUP_ERR_ARG; }
    if (ph->turb_model < ATJUP_TURB_K_EPSILON || ph->turb_model > ATJUP_TURB_K_OMEGA_SST) {
        set_error("set_physics: unknown turbulence model " + std::to_string(ph->turb_model));
        return ATJUP_ERR_ARG;
    }
    const AtjupParams& P = c->P;
    int rc = ATJUP_OK;
    auto A = [&](double** p, size_t n) { if (rc == ATJUP_OK && !*p) rc = alloc(p, n); };
    for (int s = 0; s < ATJUP_S_COUNT + 2; s++) {
        A(&c->fn[kScalarField[s]], c->NP);
        A(&c->S1[s], c->NP);
        A(&c->S2[s], c->NP);
        A(&c->Sacc[s], c->NP);
    }
    if (rc) return rc;
    if (!c->layer_h) ATJUP_CUDA(cudaMalloc(&c->layer_h, sizeof(float) * P.im));
    ATJUP_CUDA(cudaMemcpy(c->layer_h, layer_heights_km, sizeof(float) * P.im,
                          cudaMemcpyHostToDevice));
    c->phys = *ph;
    c->phys_on = (ph->species_on || ph->turb_on);
    {
        // clamp_nue's taper depth: the first level above abl_height and the one below it
        auto hm = [&](int i) {
            return ((i < 0 || i > P.im - 1) ? (double)(-1.0f) : (double)layer_heights_km[i]) * 1.0e3;
        };
        int i_abl = 0;
        while (i_abl < P.im - 1 && hm(i_abl) <= ph->abl_height) i_abl++;
        const double d = hm(std::min(i_abl, P.im - 1)) - hm(std::max(i_abl - 1, 0));
        c->turb_taper_dz = (1.0 < d) ? d : 1.0;
    }
    return ATJUP_OK;
}

int atjup_gpu_set_micro(AtjupCtx* c, const AtjupMicro* mc) {
    if (!c) { set_error("set_micro: null context"); return ATJUP_ERR_ARG; }
    if (!mc) { c->micro_on = false; return ATJUP_OK; }
    const int jm = c->P.jm;
    std::vector<double> cl(jm);
    const double pi_ = 3.14159265358979323846;
    for (int j = 0; j < jm; j++) {
        const double s = std::sin(pi_ * (double)j / (double)(jm - 1));
        cl[j] = (0.0 < s) ? s : 0.0;
    }
    if (!c->cos_lat) ATJUP_CUDA(cudaMalloc(&c->cos_lat, sizeof(double) * jm));
    ATJUP_CUDA(cudaMemcpy(c->cos_lat, cl.data(), sizeof(double) * jm, cudaMemcpyHostToDevice));
    c->micro = *mc;
    c->micro_on = true;
    return ATJUP_OK;
}

namespace {
int micro_call(AtjupCtx* c, int what, const char* name) {
    int rc = need_grid(c, name);
    if (rc) return rc;
    if (!c->micro_on || !c->phys_on) {
        set_error(std::string(name) + ": set the physics and microphysics blocks first");
        return ATJUP_ERR_ARG;
    }
    Timed tm(c, TK_MICRO);
    return launch_micro(c, what);
}
}  // namespace

int atjup_gpu_radiation(AtjupCtx* c) { return micro_call(c, MICRO_RADIATION, "radiation"); }
int atjup_gpu_precipitation(AtjupCtx* c) { return micro_call(c, MICRO_PRECIP, "precipitation"); }
int atjup_gpu_nh4sh_equilibrium(AtjupCtx* c) { return micro_call(c, MICRO_NH4SH, "nh4sh_equilibrium"); }
int atjup_gpu_diagnostics(AtjupCtx* c) { return micro_call(c, MICRO_DIAG, "diagnostics"); }
int atjup_gpu_chemistry(AtjupCtx* c) { return micro_call(c, MICRO_CHEMISTRY, "chemistry"); }
int atjup_gpu_clamp_species(AtjupCtx* c) { return micro_call(c, MICRO_CLAMP, "clamp_species"); }

int atjup_gpu_turbulence(AtjupCtx* c) {
    int rc = need_grid(c, "turbulence");
    if (rc) return rc;
    if (!c->phys_on || !c->phys.turb_on) {
        set_error("turbulence: the closure is off (atjup_gpu_set_physics with turb_on = 1 first)");
        return ATJUP_ERR_ARG;
    }
    Timed tm(c, TK_TURB);
    return launch_turbulence(c);
}

namespace {
bool is_scalar_field(int id) {
    for (int s = 0; s < ATJUP_S_COUNT + 2; s++)
        if (kScalarField[s] == id) return true;
    return false;
}
}  // namespace

int atjup_gpu_upload_n(AtjupCtx* c, int32_t id, const double* host) {
    if (!c || !host || !is_scalar_field(id) || !c->fn[id]) {
        set_error("upload_n: not a transported scalar, or physics not set");
        return ATJUP_ERR_ARG;
    }
    const size_t n = (size_t)c->P.im * c->P.jm * c->P.km;
    ATJUP_CUDA(cudaMemcpyAsync(c->stage, host, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    int rc = launch_pad(c, c->stage, c->fn[id]);
    if (rc) return rc;
    ATJUP_CUDA(cudaStreamSynchronize(c->stream));
    return ATJUP_OK;
}

int atjup_gpu_download_n(AtjupCtx* c, int32_t id, double* host) {
    if (!c || !host || !is_scalar_field(id) || !c->fn[id]) {
        set_error("download_n: not a transported scalar, or physics not set");
        return ATJUP_ERR_ARG;
    }
    const size_t n = (size_t)c->P.im * c->P.jm * c->P.km;
    int rc = launch_unpad(c, c->fn[id], c->stage);
    if (rc) return rc;
    ATJUP_CUDA(cudaMemcpyAsync(host, c->stage, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    ATJUP_CUDA(cudaStreamSynchronize(c->stream));
    return ATJUP_OK;
}

int atjup_gpu_restore_scalars(AtjupCtx* c) {
    if (!c) { set_error("restore_scalars: null context"); return ATJUP_ERR_ARG; }
    if (!c->phys_on) return ATJUP_OK;
    for (int s = 0; s < ATJUP_S_COUNT + 2; s++) {
        const int id = kScalarField[s];
        ATJUP_CUDA(cudaMemcpyAsync(c->fn[id], c->f[id], c->NP * sizeof(double),
                                   cudaMemcpyDeviceToDevice, c->stream));
    }
    return ATJUP_OK;
}

int atjup_gpu_upload2d(AtjupCtx* c, int32_t id, const double* host) {
    if (!c || !host || id < 0 || id >= ATJUP_F2_COUNT) { set_error("upload2d: bad argument"); return ATJUP_ERR_ARG; }
    ATJUP_CUDA(cudaMemcpy2DAsync(c->f2[id], c->KP * sizeof(double), host, c->P.km * sizeof(double),
                                 c->P.km * sizeof(double), c->P.jm, cudaMemcpyHostToDevice, c->stream));
    ATJUP_CUDA(cudaStreamSynchronize(c->stream));
    return ATJUP_OK;
}

int atjup_gpu_download2d(AtjupCtx* c, int32_t id, double* host) {
    if (!c || !host || id < 0 || id >= ATJUP_F2_COUNT) { set_error("download2d: bad argument"); return ATJUP_ERR_ARG; }
    ATJUP_CUDA(cudaMemcpy2DAsync(host, c->P.km * sizeof(double), c->f2[id], c->KP * sizeof(double),
                                 c->P.km * sizeof(double), c->P.jm, cudaMemcpyDeviceToHost, c->stream));
    ATJUP_CUDA(cudaStreamSynchronize(c->stream));
    return ATJUP_OK;
}

int atjup_gpu_pressure_solve(AtjupCtx* c, const AtjupSolveOpts* o, AtjupSolveStats* st) {
    int rc = need_grid(c, "pressure_solve");
    if (rc) return rc;
    AtjupSolveOpts def{};
    def.mode = ATJUP_SOLVE_SWEEPS;
    def.sweeps = c->P.press_sweeps;
    def.omega = 1.0;
    if (!o) o = &def;
    if (o->mode == ATJUP_SOLVE_RESIDUAL || o->mode == ATJUP_SOLVE_SOR) {
        Timed tm(c, TK_SOLVER);
        return pressure_residual_solve(c, o, st);
    }
    Timed tm(c, TK_PRESSURE);
    if (o->mode != ATJUP_SOLVE_SWEEPS || o->sweeps < 1) { set_error("pressure_solve: bad options"); return ATJUP_ERR_ARG; }
    if ((rc = launch_prepare_projection(c))) return rc;
    if ((rc = launch_pressure_source(c))) return rc;
    const double omega = (o->omega > 0.0) ? o->omega : 1.0;
    for (int s = 0; s < o->sweeps; s++) {
        if ((rc = launch_pressure_sweep(c, 0, omega))) return rc;
        if ((rc = launch_pressure_sweep(c, 1, omega))) return rc;
        if ((rc = launch_pressure_fold(c, c->f[ATJUP_F_P_DYN]))) return rc;
    }
    if (st) {
        st->iterations = o->sweeps; st->inner_solves = 0; st->rel_residual = -1.0; st->b_norm = -1.0;
        st->rel_floor = -1.0;
    }
    return ATJUP_OK;
}

int atjup_gpu_bc(AtjupCtx* c, int32_t which) {
    int rc = need_grid(c, "bc");
    if (rc) return rc;
    Timed tm(c, TK_BC);
    return launch_bc(c, which);
}

int atjup_gpu_shapiro(AtjupCtx* c, int32_t id, int32_t order, double strength, int32_t passes,
                      int32_t use_topo) {
    int rc = need_grid(c, "shapiro");
    if (rc) return rc;
    if (!valid_field(id) || (order != 2 && order != 4) || passes < 0) {
        set_error("shapiro: bad argument");
        return ATJUP_ERR_ARG;
    }
    Timed tm(c, TK_SHAPIRO);
    return launch_shapiro(c, c->f[id], order, strength, passes, use_topo);
}

int atjup_gpu_mixture_density(AtjupCtx* c) {
    int rc = need_grid(c, "mixture_density");
    if (rc) return rc;
    Timed tm(c, TK_MIXTURE);
    return launch_mixture_density(c);
}

int atjup_gpu_satadj(AtjupCtx* c, int32_t gas, const AtjupGasParams* gp, AtjupSatStats* stats) {
    int rc = need_grid(c, "satadj");
    if (rc) return rc;
    if (!gp || gas < ATJUP_GAS_H2O || gas > ATJUP_GAS_CH4) {
        set_error("satadj: bad argument (gas id or null parameter block)");
        return ATJUP_ERR_ARG;
    }
    {
        Timed tm(c, TK_SATADJ);
        if ((rc = launch_satadj(c, gas, *gp))) return rc;
    }
    if (stats) {
        unsigned long long h[3];
        ATJUP_CUDA(cudaMemcpyAsync(h, c->counters, sizeof h, cudaMemcpyDeviceToHost, c->stream));
        ATJUP_CUDA(cudaStreamSynchronize(c->stream));
        stats->adjusted = (int64_t)h[0];
        stats->not_converged = (int64_t)h[1];
        stats->dry_exits = (int64_t)h[2];
    }
    return ATJUP_OK;
}

int atjup_gpu_balance_column_v(AtjupCtx* c, double* vshift) {
    int rc = need_grid(c, "balance_column_v");
    if (rc) return rc;
    {
        Timed tm(c, TK_BALANCE_V);
        if ((rc = launch_balance_v(c))) return rc;
    }
    if (vshift) {
        const AtjupParams& P = c->P;
        std::vector<double> h(P.jm);
        ATJUP_CUDA(cudaMemcpyAsync(h.data(), c->dvrow, sizeof(double) * P.jm, cudaMemcpyDeviceToHost, c->stream));
        ATJUP_CUDA(cudaStreamSynchronize(c->stream));
        double m = 0.0;
        for (int j = 1; j < P.jm - 1; j++) m = std::max(m, std::fabs(h[j]));
        *vshift = m;
    }
    return ATJUP_OK;
}

namespace {
// live -> time-level-n copy of the transported scalars with the given ATJUP_S_* indices
int copy_to_n(AtjupCtx* c, const int* idx, int n) {
    for (int q = 0; q < n; q++) {
        const int id = kScalarField[idx[q]];
        ATJUP_CUDA(cudaMemcpyAsync(c->fn[id], c->f[id], c->NP * sizeof(double),
                                   cudaMemcpyDeviceToDevice, c->stream));
    }
    return ATJUP_OK;
}

// The physics part of the even iterations (cJupiterModel.cpp:1054-1162): radiation, the three
// saturation adjustments, the NH4SH equilibrium, precipitation, the scalar sync of
// ATJUP_RK_SCALAR_SYNC = 2 (t needs none: its time-level-n copy is the live field on the
// device), the closure update and the chemistry block.
int physics_block(AtjupCtx* c) {
    int rc;
    bool side_precip = false;
    const AtjupMicro& mc = c->micro;
    if (c->micro_on) {
        if (mc.radiation_on && (rc = atjup_gpu_radiation(c))) return rc;
        if (mc.satadj_on) {
            for (int g = ATJUP_GAS_H2O; g <= ATJUP_GAS_CH4; g++)
                if ((rc = atjup_gpu_satadj(c, g, &mc.gas[g], nullptr))) return rc;
        }
        if (mc.nh4sh_eq && (rc = atjup_gpu_nh4sh_equilibrium(c))) return rc;
        // Coupled precipitation writes only its sources (S_precip_*, Q_precip), which nothing
        // before the RK step reads, and reads t and the species, which nothing before the RK step
        // writes: it runs on the side stream beside the n copies, the closure update and the
        // chemistry. Uncoupled, it writes the species, and stays in order.
        side_precip = mc.precip_on && mc.precip_coupling_on;
        if (side_precip) {
            if ((rc = fork_side(c))) return rc;
            OnSide on(c);
            if ((rc = atjup_gpu_precipitation(c))) return rc;
        } else if (mc.precip_on && (rc = atjup_gpu_precipitation(c))) {
            return rc;
        }
        const int sync[11] = {ATJUP_S_H2O, ATJUP_S_H2O_CLOUD, ATJUP_S_H2O_ICE, ATJUP_S_NH3,
                              ATJUP_S_NH3_CLOUD, ATJUP_S_NH3_ICE, ATJUP_S_CH4, ATJUP_S_CH4_CLOUD,
                              ATJUP_S_CH4_ICE, ATJUP_S_H2S, ATJUP_S_NH4SH};
        if ((rc = copy_to_n(c, sync, mc.nh4sh_eq ? 11 : 9))) return rc;
    }
    if (c->phys.turb_on && (rc = atjup_gpu_turbulence(c))) return rc;
    if (c->micro_on && (rc = atjup_gpu_chemistry(c))) return rc;
    if (side_precip && (rc = join_side(c))) return rc;
    // Forces and Latent_Heat close the block (cJupiterModel.cpp:1163-1164): outputs only
    if (c->micro_on && mc.diagnostics_on && (rc = atjup_gpu_diagnostics(c))) return rc;
    return ATJUP_OK;
}
}  // namespace

int atjup_gpu_step(AtjupCtx* c, int32_t iter_n, int32_t first, const AtjupSolveOpts* solve) {
    int rc = need_grid(c, "step");
    if (rc) return rc;
    const AtjupParams& P = c->P;
    const bool ph = c->phys_on;
    if (iter_n % 2 == 0 || first) {
        if ((rc = atjup_gpu_pressure_solve(c, solve, nullptr))) return rc;
        if ((rc = atjup_gpu_mixture_density(c))) return rc;
        if (ph && (rc = physics_block(c))) return rc;
    }
    if ((rc = atjup_gpu_rk4_step(c, iter_n))) return rc;
    if ((rc = atjup_gpu_bc(c, ATJUP_BC_ALL))) return rc;
    if (ph && c->phys.turb_on) {                      // ATJUP_TURB_WALL_HOLD 1
        Timed tm(c, TK_TURB);
        if ((rc = launch_turb_wall_hold(c))) return rc;
    }
    // The moist convective adjustment reads and writes t, the vapours, condensates and tracers;
    // the velocity filters and the column balance only u, v, w: the adjustment runs on the side
    // stream beside them, joined before the species clamp.
    const bool mca_now = ph && c->mca_on && iter_n % c->mca.stride == 0;
    if (mca_now) {
        if ((rc = fork_side(c))) return rc;
        OnSide on(c);
        Timed tm(c, TK_MCA);
        if ((rc = launch_mca(c))) return rc;
    }
    if (P.shapiro_inloop > 0) {
        for (int f = ATJUP_F_U; f <= ATJUP_F_W; f++)
            if ((rc = atjup_gpu_shapiro(c, f, 4, P.shapiro_strength, P.shapiro_inloop, 1))) return rc;
    }
    if (P.v_massbal_stride > 0 && iter_n % P.v_massbal_stride == 0) {
        Timed tm(c, TK_BALANCE_V);
        if ((rc = launch_balance_v(c))) return rc;
    }
    // the flow around the obstacle re-imposed after the column balance (cJupiterModel.cpp:1362)
    if (P.cone_proj_stride > 0 && iter_n % P.cone_proj_stride == 0) {
        Timed tm(c, TK_CONE);
        if ((rc = launch_cone_projection(c))) return rc;
    }
    if (mca_now && (rc = join_side(c))) return rc;
    if (ph) {
        // clampNegativeSpecies, then restoreVar of the scalars (the dynamics need none)
        if (c->micro_on && (rc = atjup_gpu_clamp_species(c))) return rc;
        if ((rc = atjup_gpu_restore_scalars(c))) return rc;
    }
    return ATJUP_OK;
}

int atjup_gpu_nonfinite_count(AtjupCtx* c, int64_t* count) {
    if (!c || !count) return ATJUP_ERR_ARG;
    unsigned long long* d = nullptr;
    ATJUP_CUDA(cudaMalloc(&d, sizeof(unsigned long long)));
    ATJUP_CUDA(cudaMemsetAsync(d, 0, sizeof(unsigned long long), c->stream));
    int rc = launch_nonfinite(c, d);
    unsigned long long h = 0;
    if (rc == ATJUP_OK) {
        cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, c->stream);
        cudaError_t e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) rc = cuda_status(e, "nonfinite_count");
    }
    cudaFree(d);
    *count = (int64_t)h;
    if (rc == ATJUP_OK && h > 0) rc = ATJUP_ERR_NONFINITE;
    return rc;
}

int atjup_gpu_timing(AtjupCtx* c, int32_t enable) {
    if (!c) return ATJUP_ERR_ARG;
    ATJUP_CUDA(cudaStreamSynchronize(c->stream));
    c->tn = 0;
    c->tcls.clear();
    c->tgrp.clear();
    c->timing = enable != 0;
    return ATJUP_OK;
}

int atjup_gpu_timing_read(AtjupCtx* c, int32_t cls, double* total_ms, int64_t* count) {
    if (!c || cls < 0 || cls >= TK_COUNT) return ATJUP_ERR_ARG;
    double tot = 0.0;
    int64_t n = 0;
    if (cls == TK_RK_GROUP) {
        // per RK stage: from the earlier start to the later end of the dynamics kernel (slot 0)
        // and the second stream's kernels (first slot 1, last slot 2); the largest elapsed time
        // over the start and end pairs is that span
        for (size_t g = 0; g + 2 < c->tgrp.size(); g += 3) {
            const int starts[2] = {c->tgrp[g], c->tgrp[g + 1]}, ends[2] = {c->tgrp[g], c->tgrp[g + 2]};
            double span = 0.0;
            for (int en : ends) {
                if (en < 0) continue;
                ATJUP_CUDA(cudaEventSynchronize(c->tev[2 * en + 1]));
                for (int st : starts) {
                    if (st < 0) continue;
                    float ms = 0.f;
                    ATJUP_CUDA(cudaEventElapsedTime(&ms, c->tev[2 * st], c->tev[2 * en + 1]));
                    span = std::max(span, (double)ms);
                }
            }
            tot += span;
            n++;
        }
        if (total_ms) *total_ms = tot;
        if (count) *count = n;
        return ATJUP_OK;
    }
    for (int q = 0; q < c->tn; q++) {
        if (c->tcls[q] != cls) continue;
        ATJUP_CUDA(cudaEventSynchronize(c->tev[2 * q + 1]));
        float ms = 0.f;
        ATJUP_CUDA(cudaEventElapsedTime(&ms, c->tev[2 * q], c->tev[2 * q + 1]));
        tot += ms;
        n++;
    }
    if (total_ms) *total_ms = tot;
    if (count) *count = n;
    return ATJUP_OK;
}

int atjup_gpu_launch_count(AtjupCtx* c, int64_t* launches) {
    if (!c || !launches) return ATJUP_ERR_ARG;
    *launches = c->launches;
    return ATJUP_OK;
}

int atjup_gpu_synchronize(AtjupCtx* c) {
    if (!c) return ATJUP_ERR_ARG;
    ATJUP_CUDA(cudaStreamSynchronize(c->stream));
    if (int rc = xfer_synchronize(c)) return rc;
    return ATJUP_OK;
}

}  // extern "C"
