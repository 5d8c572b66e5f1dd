/*
 * Test-only harness around the unmodified ATJUP reference (RogerGrundmann/ATJUP).
 *
 * This file is TEST INFRASTRUCTURE. It is compiled together with the reference's own sources
 * (read where they lie; nothing is copied) into oracle/_ref/libatjup_ref.so by oracle/Makefile.
 * Only the test-suite, the smoke check and the CPU-baseline leg of bench.py load that library,
 * and only as the checker or as the timed reference arm -- never as the product path.
 *
 * What it adds: plain extern "C" entry points that let a caller
 *   - build a model and run the reference's own initialisation chain (cJupiterModel::Run with
 *     nm = 0: cJupiterModel.cpp:316-760 runs, the iteration loop at 1010 does not),
 *   - read / write any 3-D field as a contiguous (i, j, k) row-major block of doubles,
 *   - call one hot-path routine at a time (RungeKuttaJup, PressureSolverJup::run, the BC passes,
 *     the Shapiro filters, SaturationAdjustment, Turbulence, balanceColumnV, ...),
 *   - run one iteration of the main loop with the schedule of cJupiterModel.cpp:1032-1381.
 * The model's members are private; the harness reaches them by compiling the header with the
 * access specifiers opened up, which changes no layout.
 */
#include <algorithm>
#include <chrono>
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
#include <fcntl.h>
#include <unistd.h>
#include <sys/stat.h>
#include <sys/types.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define private public
#define protected public
#include "cJupiterModel.h"
#include "ChemistryJup.h"
#include "PressureSolverJup.h"
#include "SaturationAdjustmentJup.h"
#include "BC_Jup.h"
#include "RadiationJup.h"
#include "PrecipitationJup.h"
#include "TurbulenceJup.h"
#include "ConvectiveAdjustmentJup.h"
#include "ChromJup.h"
#undef private
#undef protected

namespace {

cJupiterModel* g_m = nullptr;
int g_saved_stdout = -1;

// Knobs that cJupiterModel.cpp reads through file-static accessors (cJupiterModel.cpp:44-52,
// 83, 86-99); the harness reads the same variables with the same defaults.
int env_i(const char* n, int d) { const char* e = getenv(n); return e ? atoi(e) : d; }
double env_d(const char* n, double d) { const char* e = getenv(n); return e ? atof(e) : d; }
int k_shapiro_inloop() { return env_i("ATJUP_VEL_SHAPIRO_INLOOP", 0); }
double k_shapiro_strength() { return env_d("ATJUP_SHAPIRO_STRENGTH", 1.0); }
int k_radiation() { return env_i("ATJUP_RADIATION", 1); }
int k_precip() { return env_i("ATJUP_PRECIP", 1); }
int k_mca_stride() { return std::max(0, env_i("ATJUP_MCA", 1)); }
int k_conv_adj() { const char* e = getenv("ATJUP_CONV_ADJ"); if (e) return atoi(e); return env_i("ATJUP_NONDIM", 0); }

Array* field_by_name(const std::string& n) {
    cJupiterModel& m = *g_m;
    static const std::map<std::string, Array cJupiterModel::*> tbl = {
#define F(x) {#x, &cJupiterModel::x}
        F(t), F(u), F(v), F(w), F(rho_mix), F(h2o), F(h2o_cloud), F(h2o_ice), F(h2s), F(nh3),
        F(nh3_cloud), F(nh3_ice), F(ch4), F(ch4_cloud), F(ch4_ice), F(nh4sh), F(chrom),
        F(tn), F(un), F(vn), F(wn), F(h2on), F(h2o_cloudn), F(h2o_icen), F(h2sn), F(nh3n),
        F(nh3_cloudn), F(nh3_icen), F(ch4n), F(ch4_cloudn), F(ch4_icen), F(nh4shn), F(chromn),
        F(massflux_h2s), F(massflux_nh3), F(massflux_nh4sh), F(difflux_h2s), F(difflux_nh3),
        F(difflux_nh4sh), F(thermalmassflux), F(p_hydro), F(p_dyn), F(p_dynn), F(p_stat),
        F(CoriolisForce), F(CentrifugalForce), F(BuoyancyForce), F(PresGradForce), F(Q_Latent),
        F(Q_Sensible),
        F(rhs_t), F(rhs_u), F(rhs_v), F(rhs_w), F(rhs_h2o), F(rhs_h2o_cloud), F(rhs_h2o_ice),
        F(rhs_h2s), F(rhs_nh3), F(rhs_nh3_cloud), F(rhs_nh3_ice), F(rhs_ch4), F(rhs_ch4_cloud),
        F(rhs_ch4_ice), F(rhs_nh4sh), F(rhs_tke), F(rhs_dis), F(acc_t), F(acc_u), F(acc_v),
        F(acc_w), F(fluxlim_nh4sh), F(aux_u), F(aux_v), F(aux_w), F(Q_rad), F(Q_precip),
        F(S_precip_h2o), F(S_precip_h2o_cloud), F(S_precip_h2o_ice), F(S_precip_nh3),
        F(S_precip_nh3_cloud), F(S_precip_nh3_ice), F(S_precip_ch4), F(S_precip_ch4_cloud),
        F(S_precip_ch4_ice), F(tke), F(tken), F(dis), F(disn), F(nue), F(prod), F(tke_source),
        F(dis_source), F(SeaMount), F(wall_nue), F(Q_Latent), F(Q_Sensible),
#undef F
    };
    auto it = tbl.find(n);
    if (it == tbl.end()) return nullptr;
    return &(m.*(it->second));
}

// The loop-local lambda turbWallOmega of cJupiterModel::Run (cJupiterModel.cpp:360-377),
// restated so a harness iteration can call it in the same places.
void turb_wall_omega(cJupiterModel& m) {
    static const int on = [](){ const char* e = getenv("ATJUP_TURB_WALL_OMEGA"); return e ? atoi(e) : 1; }();
    const char* e = getenv("ATJUP_TURB_MODEL");
    const bool k_eps = (e ? std::string(e) : m.turb_model) == "k_epsilon";
    if (on == 0 || k_eps) return;
    constexpr double nue_gas_phys = 1.8e-5;
    constexpr double bet_star = 0.09, bet_1 = 0.0333, kappa = 0.41;
    const double nd_omega = m.L_atm * 1.0e3 / m.u_0;
    for (int j = 0; j < m.jm; j++)
        for (int k = 0; k < m.km; k++) {
            const int i_w = m.surface_index(j, k);
            if (i_w <= 0 || i_w >= m.im - 1) continue;
            const double y1 = std::max(m.layer_thickness_m(std::max(i_w - 1, 0)), 1.0);
            const double y = 0.5 * y1;
            const double om_vis = 60.0 * nue_gas_phys / (bet_1 * y1 * y1);
            const double om_log = m.vel_star.y[j][k] / (std::sqrt(bet_star) * kappa * y);
            m.dis.x[i_w][j][k] = std::sqrt(om_vis * om_vis + om_log * om_log) * nd_omega;
        }
}

void gas_adjust(cJupiterModel& m, const std::string& gas) {
    if (gas == "H2O")
        SaturationAdjustmentJup(m).run("H2O", m.t_0_h2o, m.t_00_h2o, m.ep_h2o, m.lv_h2o, m.ls_h2o,
            m.C_h2o, m.L0_h2o, m.R_h2o, m.del_alf_h2o, m.del_bet_h2o,
            m.C_h2o_ice, m.L0_h2o_ice, m.del_alf_h2o_ice, m.del_bet_h2o_ice,
            m.h2o, m.h2o_cloud, m.h2o_ice);
    else if (gas == "NH3")
        SaturationAdjustmentJup(m).run("NH3", m.t_0_nh3, m.t_00_nh3, m.ep_nh3, m.lv_nh3, m.ls_nh3,
            m.C_nh3, m.L0_nh3, m.R_nh3, m.del_alf_nh3, m.del_bet_nh3,
            m.C_nh3_ice, m.L0_nh3_ice, m.del_alf_nh3_ice, m.del_bet_nh3_ice,
            m.nh3, m.nh3_cloud, m.nh3_ice);
    else if (gas == "CH4")
        SaturationAdjustmentJup(m).run("CH4", m.t_0_ch4, m.t_00_ch4, m.ep_ch4, m.lv_ch4, m.ls_ch4,
            m.C_ch4, m.L0_ch4, m.R_ch4, m.del_alf_ch4, m.del_bet_ch4,
            m.C_ch4_ice, m.L0_ch4_ice, m.del_alf_ch4_ice, m.del_bet_ch4_ice,
            m.ch4, m.ch4_cloud, m.ch4_ice);
}

// MoistConvectiveAdjustmentJup with the gases and tracers of the loop's call
// (cJupiterModel.cpp:1300-1320).
void run_mca(cJupiterModel& m) {
    typedef MoistConvectiveAdjustmentJup::Gas Gas_;
    typedef MoistConvectiveAdjustmentJup::Tracer Tr_;
    std::vector<Gas_> gases = {
        {"H2O", &m.h2o, &m.h2o_cloud, &m.h2o_ice, m.ep_h2o, m.lv_h2o, m.ls_h2o, m.t_0_h2o,
         m.C_h2o, m.L0_h2o, m.R_h2o, m.del_alf_h2o, m.del_bet_h2o, m.C_h2o_ice, m.L0_h2o_ice,
         m.del_alf_h2o_ice, m.del_bet_h2o_ice, m.t_00_h2o},
        {"NH3", &m.nh3, &m.nh3_cloud, &m.nh3_ice, m.ep_nh3, m.lv_nh3, m.ls_nh3, m.t_0_nh3,
         m.C_nh3, m.L0_nh3, m.R_nh3, m.del_alf_nh3, m.del_bet_nh3, m.C_nh3_ice, m.L0_nh3_ice,
         m.del_alf_nh3_ice, m.del_bet_nh3_ice, m.t_00_nh3}};
    const double L_nh4sh = ChemistryJup::nh4sh_eq() ? ChemistryJup::nh4sh_formation_heat() : 0.0;
    std::vector<Tr_> tracers = {{"H2S", &m.h2s, m.ep_h2s, false, 0.0},
                                {"NH4SH", &m.nh4sh, 0.0, true, L_nh4sh},
                                {"chrom", &m.chrom, 0.0, false, 0.0}};
    MoistConvectiveAdjustmentJup(m, gases, tracers).run();
}

}  // namespace

extern "C" {

// Silence (1) or restore (0) the reference's stdout chatter around harness calls.
void ref_quiet(int on) {
    fflush(stdout);
    std::cout.flush();
    if (on && g_saved_stdout < 0) {
        g_saved_stdout = dup(1);
        int fd = open("/dev/null", O_WRONLY);
        dup2(fd, 1);
        close(fd);
    } else if (!on && g_saved_stdout >= 0) {
        dup2(g_saved_stdout, 1);
        close(g_saved_stdout);
        g_saved_stdout = -1;
    }
}

// Build a model and run the reference initialisation chain (Run() with nm = 0).
// out_dir receives the reference's own init-time output files. Returns 0 on success.
int ref_create(const char* out_dir, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    if (g_m) return 1;
    g_m = new cJupiterModel();
    g_m->output_path = out_dir;
    g_m->nm = 0;
    g_m->Run();
    return 0;
}

// The stock path: build a model and run cJupiterModel::Run() with nm iterations, unchanged.
// Used to pin ref_iteration's schedule against the reference's own loop.
int ref_run_stock(const char* out_dir, int nm, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    if (g_m) return 1;
    g_m = new cJupiterModel();
    g_m->output_path = out_dir;
    g_m->nm = nm;
    g_m->Run();
    return 0;
}

void ref_set_threads(int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
}

int ref_dims(int* im, int* jm, int* km) {
    if (!g_m) return 1;
    *im = g_m->im; *jm = g_m->jm; *km = g_m->km;
    return 0;
}

// Named model scalars (resolved constants and a few knob values) for the restatement.
double ref_scalar(const char* name) {
    cJupiterModel& m = *g_m;
    const std::string n(name);
    if (n == "dt") return m.dt;
    if (n == "dr") return m.dr;
    if (n == "dthe") return m.dthe;
    if (n == "dphi") return m.dphi;
    if (n == "r_mix") return m.r_mix;
    if (n == "R_mix") return m.R_mix;
    if (n == "cp_mix") return m.cp_mix;
    if (n == "mue_mix") return m.mue_mix;
    if (n == "u_0") return m.u_0;
    if (n == "t_ref") return m.t_ref;
    if (n == "L_atm") return m.L_atm;
    if (n == "g") return m.g;
    if (n == "omega") return m.omega;
    if (n == "re") return m.re;
    if (n == "pr") return m.pr;
    if (n == "Coriolis") return m.Coriolis;
    if (n == "centrifugal") return m.centrifugal;
    if (n == "buoyancy") return m.buoyancy;
    if (n == "chemical_reaction") return m.chemical_reaction;
    if (n == "p_dyn_to_bar") return m.p_dyn_to_bar();
    if (n == "sinthe_min") return cJupiterModel::sinthe_min();
    if (n == "t_diff_scale") return cJupiterModel::t_diff_scale();
    if (n == "species_diff_scale") return cJupiterModel::species_diff_scale();
    if (n == "coord_stretching") return m.coord_stretching ? 1.0 : 0.0;
    if (n == "use_turbulence_model") return m.use_turbulence_model ? 1.0 : 0.0;
    if (n == "cell_hold") return (cJupiterModel::cell_hold() && !m.cell_vbar0.empty()) ? 1.0 : 0.0;
    if (n == "metric_split") return cJupiterModel::metric_split() ? 1.0 : 0.0;
    if (n == "coriolis_split") return cJupiterModel::coriolis_split() ? 1.0 : 0.0;
    if (n == "geo_balance") return cJupiterModel::geo_balance() ? 1.0 : 0.0;
    if (n == "has_p_baro") return m.p_baro.empty() ? 0.0 : 1.0;
    if (n == "iter_n") return m.iter_n;
    if (n == "re_turb") return m.re_turb;
    if (n == "ep_h2s") return m.ep_h2s;
    if (n == "sc_h2o") return m.sc_h2o;
    if (n == "sc_h2s") return m.sc_h2s;
    if (n == "sc_nh3") return m.sc_nh3;
    if (n == "sc_ch4") return m.sc_ch4;
    if (n == "sc_nh4sh") return m.sc_nh4sh;
    if (n == "rg_nh4sh") return m.rg_nh4sh;
    if (n == "r_p_nh4sh") return m.r_p_nh4sh;
    if (n == "m_nh3") return m.m_nh3;
    if (n == "m_h2s") return m.m_h2s;
    if (n == "m_nh4sh") return m.m_nh4sh;
    if (n == "D_nh3") return m.mue_nh3 / (m.rg_nh3 * m.sc_nh3);
    if (n == "D_h2s") return m.mue_h2s / (m.rg_h2s * m.sc_h2s);
    if (n == "D_nh4sh") return m.mue_nh4sh / (m.rg_nh4sh * m.sc_nh4sh);
    if (n == "polar_divisor_floor") return ATPhys::polar_divisor_floor<cJupiterModel>();
    if (n == "coeff_h2o_A") return m.coeff_h2o_A;
    if (n == "coeff_h2o_B") return m.coeff_h2o_B;
    if (n == "coeff_h2o_A_i") return m.coeff_h2o_A_i;
    if (n == "coeff_h2o_B_i") return m.coeff_h2o_B_i;
    if (n == "coeff_nh3_A") return m.coeff_nh3_A;
    if (n == "coeff_nh3_B") return m.coeff_nh3_B;
    if (n == "coeff_nh3_A_i") return m.coeff_nh3_A_i;
    if (n == "coeff_nh3_B_i") return m.coeff_nh3_B_i;
    if (n == "t_0_nh4sh") return m.t_0_nh4sh;
    if (n == "t_00_nh4sh") return m.t_00_nh4sh;
    if (n == "rad_F_int") return cJupiterModel::rad_F_int();
    if (n == "rad_S_solar") return cJupiterModel::rad_S_solar();
    if (n == "rad_albedo_bond") return cJupiterModel::rad_albedo_bond();
    if (n == "rad_x_H2") return cJupiterModel::rad_x_H2();
    if (n == "rad_x_He") return cJupiterModel::rad_x_He();
    if (n == "rad_cia_strength") return ATPhys::env_double("ATJUP", "CIA_STRENGTH", cJupiterModel::rad_default_cia_strength());
    if (n == "rad_opacity_strength") return ATPhys::env_double("ATJUP", "OPACITY_STRENGTH", 1.0);
    if (n == "rad_solar") return ATPhys::env_int("ATJUP", "SOLAR", 1);
    if (n == "rad_solar_strength") return ATPhys::env_double("ATJUP", "SOLAR_STRENGTH", 1.0);
    if (n == "rad_sw_tau_per_bar") return ATPhys::env_double("ATJUP", "SW_TAU_PER_BAR", 1.0);
    if (n == "rad_bottom") return ATPhys::env_int("ATJUP", "RAD_BOTTOM", cJupiterModel::rad_default_bottom());
    if (n == "precip_rate_scale") return PrecipitationJup::rate_scale();
    if (n == "precip_coupling_on") return PrecipitationJup::coupling_on() ? 1.0 : 0.0;
    return std::nan("");
}

int ref_get3(const char* name, double* out) {
    Array* a = field_by_name(name);
    if (!a) return 1;
    const int im = g_m->im, jm = g_m->jm, km = g_m->km;
    for (int i = 0; i < im; i++)
        for (int j = 0; j < jm; j++)
            std::memcpy(out + ((size_t)i * jm + j) * km, a->x[i][j], sizeof(double) * km);
    return 0;
}

int ref_set3(const char* name, const double* in) {
    Array* a = field_by_name(name);
    if (!a) return 1;
    const int im = g_m->im, jm = g_m->jm, km = g_m->km;
    for (int i = 0; i < im; i++)
        for (int j = 0; j < jm; j++)
            std::memcpy(a->x[i][j], in + ((size_t)i * jm + j) * km, sizeof(double) * km);
    return 0;
}

// 1-D and flattened vectors: rad, the, phi, buoy_ref_level, cell_vbar0, cell_ubar0, p_baro,
// layer_heights (float in the model, widened), vel_star (jm*km). Returns the element count,
// or -1 for an unknown name; copies at most cap elements.
int ref_get1(const char* name, double* out, int cap) {
    cJupiterModel& m = *g_m;
    const std::string n(name);
    std::vector<double> v;
    if (n == "rad") v.assign(m.rad.z, m.rad.z + m.im);
    else if (n == "the") v.assign(m.the.z, m.the.z + m.jm);
    else if (n == "phi") v.assign(m.phi.z, m.phi.z + m.km);
    else if (n == "buoy_ref_level") v = m.buoy_ref_level;
    else if (n == "cell_vbar0") v = m.cell_vbar0;
    else if (n == "cell_ubar0") v = m.cell_ubar0;
    else if (n == "p_baro") v = m.p_baro;
    else if (n == "layer_heights") for (float f : m.m_layer_heights) v.push_back((double)f);
    else if (n == "vel_star") {
        for (int j = 0; j < m.jm; j++) for (int k = 0; k < m.km; k++) v.push_back(m.vel_star.y[j][k]);
    } else return -1;
    const int nn = (int)v.size();
    for (int q = 0; q < std::min(nn, cap); q++) out[q] = v[q];
    return nn;
}

int ref_get_topo(int* out) {
    cJupiterModel& m = *g_m;
    for (int j = 0; j < m.jm; j++)
        for (int k = 0; k < m.km; k++) out[(size_t)j * m.km + k] = m.i_topography[j][k];
    return 0;
}

void ref_set_iter(int iter_n) { g_m->iter_n = iter_n; }
// the model object, for the drop-in harness compiled beside this one (gpu_dropin.cpp)
void* ref_model_ptr(void) { return g_m; }

// ---- single hot-path routines ----
void ref_rk4() { g_m->RungeKuttaJup(); }
void ref_buoy_ref_level() { g_m->computeBuoyancyRefLevel(); }
void ref_hydrostatic() { g_m->computeHydrostaticPressure(false); }
void ref_pressure() { PressureSolverJup(*g_m).run(); }
void ref_prepare_projection(int rigid) { g_m->prepareProjectionBoundaries(rigid != 0); }
void ref_bc_radius() { BC_Jup(*g_m).bcRadius(); }
void ref_bc_theta() { BC_Jup(*g_m).bcTheta(); }
void ref_bc_phi() { BC_Jup(*g_m).bcPhi(); }
void ref_bc_solid() { BC_Jup(*g_m).bcSolidGround(); }
double ref_balance_v() { return g_m->balanceColumnV(nullptr); }
void ref_clamp_species() { g_m->clampNegativeSpecies(); }
void ref_radiation() { RadiationJup(*g_m).run(); }
void ref_precipitation() { PrecipitationJup(*g_m).run(); }
void ref_nh4sh_eq() { ChemistryJup(*g_m).EquilibriumNH4SH("loop"); }
// the output diagnostics that close the physics block (cJupiterModel.cpp:1163-1164)
void ref_diagnostics() { g_m->Forces(); g_m->Latent_Heat(); }
// The chemistry block of the loop (cJupiterModel.cpp:1144-1162 in the order ref_iteration runs
// it): diffusive fluxes, their 1-2-1 smoothing, the mass rate, the NH4SH flux limiter and the
// smoothing of the mass fluxes.
void ref_chem_fluxes() {
    cJupiterModel& m = *g_m;
    ChemistryJup(m).DiffMassFluxJup();
    JupiterUtils::damp_wiggles(m.difflux_h2s, &m.i_topography, true, true, true);
    JupiterUtils::damp_wiggles(m.difflux_nh3, &m.i_topography, true, true, true);
    JupiterUtils::damp_wiggles(m.difflux_nh4sh, &m.i_topography, true, true, true);
    JupiterUtils::damp_wiggles(m.thermalmassflux, &m.i_topography, true, true, true);
    ChemistryJup(m).ChemMassRateJup();
    ChemistryJup(m).FluxLimiterNH4SH();
    JupiterUtils::damp_wiggles(m.massflux_h2s, &m.i_topography, true, true, true);
    JupiterUtils::damp_wiggles(m.massflux_nh3, &m.i_topography, true, true, true);
    JupiterUtils::damp_wiggles(m.massflux_nh4sh, &m.i_topography, true, true, true);
    JupiterUtils::damp_wiggles(m.fluxlim_nh4sh, &m.i_topography, true, true, true);
}
void ref_restore() { g_m->restoreVar(1.0); }
void ref_mca() { run_mca(*g_m); }

// cJupiterModel::save_state / load_state (FileIO_Jup.cpp:584-683) with the model's output
// directory pointed at dir for the call: the file is dir/jup_restart_<iter>.bin.
int ref_save_state(const char* dir, int iter) {
    const std::string keep = g_m->output_path;
    g_m->output_path = dir;
    g_m->save_state(iter);
    g_m->output_path = keep;
    return 0;
}
int ref_load_state(const char* dir, int iter) {
    const std::string keep = g_m->output_path;
    g_m->output_path = dir;
    const bool ok = g_m->load_state(iter);
    g_m->output_path = keep;
    return ok ? 0 : 1;
}
void ref_mixture_density() { g_m->computeMixtureDensity(); }
// the in-loop projection of the flow around the obstacle (cJupiterModel.cpp:1362-1363)
// one in-loop projection around the obstacle (InitValues_Jup.cpp:1595-1822); with verbose its
// summary line (SOR iterations up to N, wall inflow, divergence) is printed and flushed
void ref_cone_proj(int verbose) {
    g_m->projectAroundObstacle(true, verbose != 0);
    fflush(stdout);
}
void ref_satadj(const char* gas) { gas_adjust(*g_m, gas); }

// The 14 per-gas constants cJupiterModel passes to SaturationAdjustmentJup::run
// (cJupiterModel.cpp:1060-1080), in the order of SaturationAdjustment.h:236-243:
// t_0, t_00, ep, lv, ls, C, L0, R, del_alf, del_bet, C_i, L0_i, del_alf_i, del_bet_i.
int ref_gas_consts(const char* gas, double* out) {
    cJupiterModel& m = *g_m;
    const std::string g(gas);
#define G(s) { const double v[14] = {m.t_0_##s, m.t_00_##s, m.ep_##s, m.lv_##s, m.ls_##s, \
        m.C_##s, m.L0_##s, m.R_##s, m.del_alf_##s, m.del_bet_##s, m.C_##s##_ice, m.L0_##s##_ice, \
        m.del_alf_##s##_ice, m.del_bet_##s##_ice}; std::memcpy(out, v, sizeof v); return 0; }
    if (g == "H2O") G(h2o)
    if (g == "NH3") G(nh3)
    if (g == "CH4") G(ch4)
#undef G
    return 1;
}
void ref_turbulence() { TurbulenceJup(*g_m).run(); turb_wall_omega(*g_m); }

// One Shapiro filter call on a named field: order 2 = damp_wiggles, 4 = damp_wiggles_ho
// (lib/Utils.cpp:227-453), with the model's i_topography as the fluid floor when use_topo.
int ref_shapiro(const char* name, int order, double strength, int passes, int use_topo) {
    Array* a = field_by_name(name);
    if (!a) return 1;
    const std::vector<std::vector<int>>* topo = use_topo ? &g_m->i_topography : nullptr;
    if (order == 4) JupiterUtils::damp_wiggles_ho(*a, topo, true, true, true, strength, passes);
    else JupiterUtils::damp_wiggles(*a, topo, true, true, true, strength, passes);
    return 0;
}

/*
 * One iteration of the main loop, in the order of cJupiterModel.cpp:1032-1381. Print-only
 * diagnostics are left out. `dry` = 1 skips the saturation adjustment, the NH4SH equilibrium and
 * the chemistry mass-flux block (the reference has no switch for these; with the species zeroed
 * they have nothing to act on). Returns nonzero if a knob asks for a routine the harness does not
 * call (moist convective adjustment, dry convective adjustment).
 */
int ref_iteration(int iter_n, int first, int dry) {
    cJupiterModel& m = *g_m;
    m.iter_n = iter_n;
    if (k_conv_adj()) return 2;
    if (iter_n % 2 == 0 || first) {
        PressureSolverJup(m).run();
        static const bool damp_pdyn = [](){ const char* e = getenv("ATJUP_DAMP_PDYN"); return e ? atoi(e) != 0 : !cJupiterModel::geo_balance(); }();
        if (damp_pdyn) JupiterUtils::damp_wiggles(m.p_dyn, &m.i_topography, true, true, true);
        m.computeMixtureDensity();
        if (k_radiation()) RadiationJup(m).run();
        if (!dry) {
            gas_adjust(m, "H2O");
            gas_adjust(m, "NH3");
            gas_adjust(m, "CH4");
            if (ChemistryJup::nh4sh_eq()) ChemistryJup(m).EquilibriumNH4SH("loop");
        }
        if (k_precip()) PrecipitationJup(m).run();
        static const int rk_scalar_sync = [](){ const char* e = getenv("ATJUP_RK_SCALAR_SYNC"); return e ? atoi(e) : 2; }();
        const bool nh4sh_sync = ChemistryJup::nh4sh_eq();
        if (rk_scalar_sync >= 1) {
            for (int i = 0; i < m.im; i++)
                for (int j = 0; j < m.jm; j++)
                    for (int k = 0; k < m.km; k++) {
                        m.h2on.x[i][j][k] = m.h2o.x[i][j][k];
                        m.h2o_cloudn.x[i][j][k] = m.h2o_cloud.x[i][j][k];
                        m.h2o_icen.x[i][j][k] = m.h2o_ice.x[i][j][k];
                        m.nh3n.x[i][j][k] = m.nh3.x[i][j][k];
                        m.nh3_cloudn.x[i][j][k] = m.nh3_cloud.x[i][j][k];
                        m.nh3_icen.x[i][j][k] = m.nh3_ice.x[i][j][k];
                        m.ch4n.x[i][j][k] = m.ch4.x[i][j][k];
                        m.ch4_cloudn.x[i][j][k] = m.ch4_cloud.x[i][j][k];
                        m.ch4_icen.x[i][j][k] = m.ch4_ice.x[i][j][k];
                        if (rk_scalar_sync >= 2) m.tn.x[i][j][k] = m.t.x[i][j][k];
                        if (nh4sh_sync) { m.h2sn.x[i][j][k] = m.h2s.x[i][j][k]; m.nh4shn.x[i][j][k] = m.nh4sh.x[i][j][k]; }
                    }
        }
        if (m.use_turbulence_model) { TurbulenceJup(m).run(); turb_wall_omega(m); }
        if (!dry) {
            ChemistryJup(m).DiffMassFluxJup();
            JupiterUtils::damp_wiggles(m.difflux_h2s, &m.i_topography, true, true, true);
            JupiterUtils::damp_wiggles(m.difflux_nh3, &m.i_topography, true, true, true);
            JupiterUtils::damp_wiggles(m.difflux_nh4sh, &m.i_topography, true, true, true);
            JupiterUtils::damp_wiggles(m.thermalmassflux, &m.i_topography, true, true, true);
            ChemistryJup(m).ChemMassRateJup();
            ChemistryJup(m).FluxLimiterNH4SH();
            JupiterUtils::damp_wiggles(m.massflux_h2s, &m.i_topography, true, true, true);
            JupiterUtils::damp_wiggles(m.massflux_nh3, &m.i_topography, true, true, true);
            JupiterUtils::damp_wiggles(m.massflux_nh4sh, &m.i_topography, true, true, true);
            JupiterUtils::damp_wiggles(m.fluxlim_nh4sh, &m.i_topography, true, true, true);
            m.Forces();
            m.Latent_Heat();
        }
    }
    m.chromUV();
    m.RungeKuttaJup();
    BC_Jup(m).bcRadius();
    BC_Jup(m).bcTheta();
    BC_Jup(m).bcPhi();
    BC_Jup(m).bcSolidGround();
    static const int turb_wall_hold = [](){ const char* e = getenv("ATJUP_TURB_WALL_HOLD"); return e ? atoi(e) : 1; }();
    if (m.use_turbulence_model && turb_wall_hold != 0) { TurbulenceJup(m).apply_wall_bc(); turb_wall_omega(m); }
    if (k_mca_stride() > 0 && iter_n % k_mca_stride() == 0) run_mca(m);
    if (k_shapiro_inloop() > 0) {
        const double s = k_shapiro_strength();
        JupiterUtils::damp_wiggles_ho(m.u, &m.i_topography, true, true, true, s, k_shapiro_inloop());
        JupiterUtils::damp_wiggles_ho(m.v, &m.i_topography, true, true, true, s, k_shapiro_inloop());
        JupiterUtils::damp_wiggles_ho(m.w, &m.i_topography, true, true, true, s, k_shapiro_inloop());
    }
    if (cJupiterModel::v_massbal_stride() > 0 && iter_n % cJupiterModel::v_massbal_stride() == 0)
        m.balanceColumnV(nullptr);
    if (cJupiterModel::cone_proj_stride() > 0 && iter_n % cJupiterModel::cone_proj_stride() == 0)
        m.projectAroundObstacle(true, false);
    m.clampNegativeSpecies();
    m.restoreVar(1.0);
    return 0;
}

// Knob values that select branches of the hot path, for the restatement's parameter block.
int ref_knob(const char* name) {
    cJupiterModel& m = *g_m;
    const std::string n(name);
    if (n == "shapiro_vel_inloop") return k_shapiro_inloop();
    if (n == "v_massbal_stride") return cJupiterModel::v_massbal_stride();
    if (n == "cone_proj_stride") return cJupiterModel::cone_proj_stride();
    if (n == "mca_stride") return k_mca_stride();
    if (n == "radiation") return k_radiation();
    if (n == "precip") return k_precip();
    if (n == "phi_periodic") return ATPhys::phi_periodic<cJupiterModel>() ? 1 : 0;
    if (n == "nh4sh_eq") return ChemistryJup::nh4sh_eq() ? 1 : 0;
    if (n == "local_rho") return cJupiterModel::local_rho() ? 1 : 0;
    if (n == "turb_model") {   // TurbulenceJup's parse: k_epsilon 0, k_omega 1, anything else SST 2
        const char* e = getenv("ATJUP_TURB_MODEL");
        const std::string t = e ? std::string(e) : m.turb_model;
        return t == "k_epsilon" ? 0 : (t == "k_omega" ? 1 : 2);
    }
    if (n == "turb_buoy") { const char* e = getenv("ATJUP_TURB_BUOY"); return e ? atoi(e) : 0; }
    if (n == "nh4sh_cap") { const char* e = getenv("ATJUP_NH4SH_CAP"); return e ? atoi(e) : 0; }
    if (n == "t_limiter") { const char* e = getenv("ATJUP_T_LIMITER"); return e ? atoi(e) : 0; }
    if (n == "rk_scalar_sync") { const char* e = getenv("ATJUP_RK_SCALAR_SYNC"); return e ? atoi(e) : 2; }
    return -999;
}
double ref_knob_d(const char* name) {
    cJupiterModel& m = *g_m;
    const std::string n(name);
    if (n == "shapiro_strength") return k_shapiro_strength();
    if (n == "nue_max_phys") return TurbulenceJup::nue_max_phys();
    if (n == "tke_max") { const char* e = getenv("ATJUP_TKE_MAX"); return e ? atof(e) : 1000.0; }
    if (n == "turb_buoy_prt") { const char* e = getenv("ATJUP_TURB_BUOY_PRT"); return e ? atof(e) : 0.9; }
    if (n == "species_divu") { const char* e = getenv("ATJUP_SPECIES_DIVU"); return e ? atof(e) : 0.0; }
    if (n == "abl_height") return m.abl_height;
    if (n == "turb_free") return TurbulenceJup::turb_free();
    if (n == "turb_k_bg") return TurbulenceJup::turb_k_bg();
    if (n == "turb_clamp_pass") return TurbulenceJup::turb_clamp_pass();
    return std::nan("");
}

}  // extern "C"
