// Boundary passes after the RK step, over the dynamics fields and, with the physics on, the
// species, the chemistry mass fluxes and the closure fields.
//
// Reference: BC_Jup::bcRadius (BC_Jup.h:185-263) around BoundaryConditions<M>::bcRadius
// (BoundaryConditions.h:151-250), bcTheta (253-336), bcPhi (339-360, periodic seam), and
// BC_Jup::bcSolidGround (BC_Jup.h:460-658). Each pass is independent per boundary row or column,
// so each is one kernel over that 2-D face; the solid-cell pass walks a list of the obstacle's
// cells (with their extrapolation partners) built once from the static mask.
#include "ctx.cuh"

namespace atjup {
namespace {

constexpr double kC43 = 4.0 / 3.0, kC13 = 1.0 / 3.0;

// Zonal means of v and w at levels im-3 and im-2 over the km-1 distinct meridians, taken before
// the radial pass for the zonal-mean-preserving sponge (ATJUP_BC_TOP_TAPER = 3).
__global__ void zonal_mean_kernel(const double* __restrict__ v, const double* __restrict__ w,
                                  double* __restrict__ zm, int im, int jm, int km, int KP) {
    const int j = blockIdx.x, l = blockIdx.y;
    const int i = im - 3 + l;
    const size_t b = ((size_t)i * jm + j) * KP;
    double sv = 0.0, sw = 0.0;
    for (int k = threadIdx.x; k < km - 1; k += 32) { sv += v[b + k]; sw += w[b + k]; }
    for (int o = 16; o > 0; o >>= 1) {
        sv += __shfl_down_sync(0xffffffffu, sv, o);
        sw += __shfl_down_sync(0xffffffffu, sw, o);
    }
    if (threadIdx.x == 0) {
        zm[(size_t)(2 * l) * jm + j] = sv / (km - 1);
        zm[(size_t)(2 * l + 1) * jm + j] = sw / (km - 1);
    }
}

// A list of fields a pass treats alike (the reference's bc_fields_* lists, BC_Jup.h:275-350).
struct FieldList {
    double* f[32];
    int n;
};

// One (j, k) column: 2-point Neumann at both radial walls for every listed field
// (BoundaryConditions.h:176-193), the rigid lid u = 0, the top taper of v, w (taper 3: zonal-mean
// preserving, BC_Jup.h:186-229), then the species wall copy at i = 0 and positivity at both
// walls (BC_Jup.h:231-262). Each step is column-local, so doing them per column in the
// reference's order equals the reference's sequence of whole-grid passes.
__global__ void radius_kernel(FieldList L, FieldList Q, double* __restrict__ u,
                              double* __restrict__ v, double* __restrict__ w,
                              const double* __restrict__ zm, int im, int jm, int km, int KP,
                              int lid_u, int taper) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (k >= km) return;
    const size_t plane = (size_t)jm * KP, b = (size_t)j * KP + k;
    for (int f = 0; f < L.n; f++) {
        double* x = L.f[f];
        x[b] = kC43 * x[b + plane] - kC13 * x[b + 2 * plane];
        x[b + (im - 1) * plane] = kC43 * x[b + (im - 2) * plane] - kC13 * x[b + (im - 3) * plane];
    }
    if (lid_u) {
        u[b] = 0.0;
        u[b + (im - 1) * plane] = 0.0;
    }
    const size_t c1 = b + (im - 1) * plane, c2 = b + (im - 2) * plane, c3 = b + (im - 3) * plane;
    if (taper != 0) {
        v[c1] = 0.0;
        w[c1] = 0.0;
        if (taper == 2) {
            const size_t c4 = b + (im - 4) * plane;
            v[c2] = (1.0 / 3.0) * v[c4];
            w[c2] = (1.0 / 3.0) * w[c4];
            v[c3] = (2.0 / 3.0) * v[c4];
            w[c3] = (2.0 / 3.0) * w[c4];
        } else {
            v[c2] *= (1.0 / 3.0);
            w[c2] *= (1.0 / 3.0);
            v[c3] *= (2.0 / 3.0);
            w[c3] *= (2.0 / 3.0);
        }
    }
    if (taper == 3) {
        const double v3 = zm[j], w3 = zm[jm + j], v2 = zm[2 * jm + j], w2 = zm[3 * jm + j];
        v[c3] += (1.0 / 3.0) * v3;
        w[c3] += (1.0 / 3.0) * w3;
        v[c2] += (2.0 / 3.0) * v2;
        w[c2] += (2.0 / 3.0) * w2;
        v[c1] = v2;
        w[c1] = w2;
    }
    for (int f = 0; f < Q.n; f++) {
        double* x = Q.f[f];
        double x0 = x[b + plane];                  // wall copy
        if (x0 < 0.0) x0 = 0.0;                    // positivity
        x[b] = x0;
        if (x[c1] < 0.0) x[c1] = 0.0;
    }
}

// Pole rows (BoundaryConditions.h:253-336): rows 1..nfill copy row nfill+1 for the extrapolated
// list and ramp r/(nfill+1) of it for the zero list; the pole row copies row 1 (extrapolated
// list) or is zero (zero list).
__global__ void theta_kernel(FieldList X, FieldList Z, int im, int jm, int km, int KP, int nfill) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (k >= km) return;
    const size_t b = (size_t)i * jm * KP + k;
    auto at = [&](int jj) { return b + (size_t)jj * KP; };
    if (nfill > 0) {
        const int jf = nfill + 1;
        for (int r = 1; r <= nfill; r++) {
            const double ramp = (double)r / (double)jf;
            for (int f = 0; f < X.n; f++) {
                double* x = X.f[f];
                x[at(r)] = x[at(jf)];
                x[at(jm - 1 - r)] = x[at(jm - 1 - jf)];
            }
            for (int f = 0; f < Z.n; f++) {
                double* x = Z.f[f];
                x[at(r)] = ramp * x[at(jf)];
                x[at(jm - 1 - r)] = ramp * x[at(jm - 1 - jf)];
            }
        }
    }
    for (int f = 0; f < Z.n; f++) {
        Z.f[f][at(0)] = 0.0;
        Z.f[f][at(jm - 1)] = 0.0;
    }
    for (int f = 0; f < X.n; f++) {
        double* x = X.f[f];
        x[at(0)] = x[at(1)];
        x[at(jm - 1)] = x[at(jm - 2)];
    }
}

__global__ void phi_kernel(FieldList L, int jm, int km, int KP) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (j >= jm) return;
    const size_t b = ((size_t)i * jm + j) * KP;
    for (int f = 0; f < L.n; f++) L.f[f][b + km - 1] = L.f[f][b];
}

// Solid cells (BC_Jup.h:496-590): velocities 0; surface cells with an extrapolation pair take
// the 2-point extrapolation of every listed scalar; the others set the list from index 2 (p_dyn)
// on to 0, keeping t and p_stat.
__global__ void solid_kernel(const SolidCell* __restrict__ Ls, int n, FieldList S,
                             double* __restrict__ u, double* __restrict__ v,
                             double* __restrict__ w) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const SolidCell s = Ls[q];
    u[s.c] = 0.0;
    v[s.c] = 0.0;
    w[s.c] = 0.0;
    if (s.kind == 1) {
        for (int f = 0; f < S.n; f++) S.f[f][s.c] = kC43 * S.f[f][s.a] - kC13 * S.f[f][s.b];
    } else {
        for (int f = 2; f < S.n; f++) S.f[f][s.c] = 0.0;
    }
}

__device__ __forceinline__ double safe_clamp(double v, double lo, double hi) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    if ((b & 0x7FF0000000000000ULL) == 0x7FF0000000000000ULL) return lo;
    return (v < lo) ? lo : ((v > hi) ? hi : v);
}

// The sanitising clamps of the closure fields over the whole grid (BC_Jup.h:627-655), with the
// fixed bounds of that routine: k* in [0, 1000 m2/s2], omega* in [1e-10, 1e6], nue* in
// [0, 1e5 m2/s], prod in [0, 1e4], sources in [-1e4, 1e4]; NaN and Inf go to the lower bound.
struct SanArgs {
    double *tke, *tken, *dis, *disn, *nue, *prod, *tsrc, *dsrc;
    size_t n;
    double tke_max, nue_max;
};
__global__ void sanitise_kernel(SanArgs a) {
    const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.n) return;
    const double prod_max = 1.0e4, dis_max = 1.0e6;
    a.tke[c] = safe_clamp(a.tke[c], 0.0, a.tke_max);
    a.tken[c] = safe_clamp(a.tken[c], 0.0, a.tke_max);
    a.dis[c] = safe_clamp(a.dis[c], 1.0e-10, dis_max);
    a.disn[c] = safe_clamp(a.disn[c], 1.0e-10, dis_max);
    a.nue[c] = safe_clamp(a.nue[c], 0.0, a.nue_max);
    a.prod[c] = safe_clamp(a.prod[c], 0.0, prod_max);
    a.tsrc[c] = safe_clamp(a.tsrc[c], -prod_max, prod_max);
    a.dsrc[c] = safe_clamp(a.dsrc[c], -prod_max, prod_max);
}

// Ambient temperature of the solid cells of one (i, j) row: the mean of t over its fluid cells.
__global__ void ambient_kernel(const int32_t* __restrict__ rows, const uint8_t* __restrict__ s,
                               double* __restrict__ t, int jm, int km, int KP) {
    const int r = rows[blockIdx.x];
    const size_t b = (size_t)r * KP;
    double sum = 0.0;
    int n = 0;
    for (int k = threadIdx.x; k < km; k += 32)
        if (!s[b + k]) { sum += t[b + k]; n++; }
    for (int o = 16; o > 0; o >>= 1) {
        sum += __shfl_down_sync(0xffffffffu, sum, o);
        n += __shfl_down_sync(0xffffffffu, n, o);
    }
    sum = __shfl_sync(0xffffffffu, sum, 0);
    n = __shfl_sync(0xffffffffu, n, 0);
    if (n == 0) return;
    const double t_amb = sum / n;
    for (int k = threadIdx.x; k < km; k += 32)
        if (s[b + k]) t[b + k] = t_amb;
}

}  // namespace

int launch_bc(AtjupCtx* c, int which) {
    return launch_bc_ptrs(c, which, c->f[ATJUP_F_T], c->f[ATJUP_F_U], c->f[ATJUP_F_V],
                          c->f[ATJUP_F_W], c->f[ATJUP_F_P_DYN], c->f[ATJUP_F_P_STAT], c->phys_on);
}

// The passes on the given t, u, v, w, p_dyn, p_stat (the dry lists unless phys, which takes the
// context's other fields as well): the tangent-linear of the dry passes is this on perturbations.
int launch_bc_ptrs(AtjupCtx* c, int which, double* t, double* u, double* v, double* w,
                   double* p_dyn, double* p_stat, bool phys) {
    const AtjupParams& P = c->P;
    const bool ph = phys;
    // the field lists of the passes (BC_Jup.h:275-350) over the fields the device holds
    auto add = [](FieldList& L, double* x) { L.f[L.n++] = x; };
    auto add_species = [&](FieldList& L) {
        for (int s = 0; s < ATJUP_S_COUNT; s++) add(L, c->f[kScalarField[s]]);
    };
    auto add_turb = [&](FieldList& L) {
        add(L, c->f[ATJUP_F_TKE]); add(L, c->f[ATJUP_F_DIS]); add(L, c->f[ATJUP_F_NUE]);
        add(L, c->f[ATJUP_F_PROD]); add(L, c->f[ATJUP_F_TKE_SOURCE]); add(L, c->f[ATJUP_F_DIS_SOURCE]);
    };
    auto add_massflux = [&](FieldList& L, bool fluxlim) {
        add(L, c->f[ATJUP_F_MASSFLUX_H2S]); add(L, c->f[ATJUP_F_MASSFLUX_NH3]);
        add(L, c->f[ATJUP_F_MASSFLUX_NH4SH]);
        if (fluxlim) add(L, c->f[ATJUP_F_FLUXLIM_NH4SH]);
        // the diffusive fluxes travel with the mass fluxes in every list that has them
        add(L, c->f[ATJUP_F_DIFFLUX_H2S]); add(L, c->f[ATJUP_F_DIFFLUX_NH3]);
        add(L, c->f[ATJUP_F_DIFFLUX_NH4SH]);
    };
    if (which & ATJUP_BC_RADIUS) {
        FieldList L{}, Q{};
        add(L, t); add(L, u); add(L, v); add(L, w);
        if (ph) { add_species(L); add_massflux(L, false); add_turb(L); add_species(Q); }
        if (P.top_taper == 3) {
            c->launches++;
            zonal_mean_kernel<<<dim3(P.jm, 2), 32, 0, c->stream>>>(v, w, c->zm, P.im, P.jm, P.km, c->KP);
        }
        c->launches++;
        radius_kernel<<<dim3((P.km + 127) / 128, P.jm), 128, 0, c->stream>>>(
            L, Q, u, v, w, c->zm, P.im, P.jm, P.km, c->KP, P.lid_u, P.top_taper);
        ATJUP_CHECK_LAUNCH("bc_radius");
    }
    if (which & ATJUP_BC_THETA) {
        FieldList X{}, Z{};
        add(X, t); add(X, u);
        add(Z, v); add(Z, w);
        if (ph) { add_species(X); add_turb(X); add_massflux(Z, true); }
        c->launches++;
        theta_kernel<<<dim3((P.km + 127) / 128, P.im), 128, 0, c->stream>>>(
            X, Z, P.im, P.jm, P.km, c->KP, P.pole_fill_rows);
        ATJUP_CHECK_LAUNCH("bc_theta");
    }
    if (which & ATJUP_BC_PHI) {
        FieldList L{};
        add(L, t); add(L, u); add(L, v); add(L, w);
        if (ph) { add_species(L); add_massflux(L, true); add_turb(L); }
        c->launches++;
        phi_kernel<<<dim3((P.jm + 127) / 128, P.im), 128, 0, c->stream>>>(L, P.jm, P.km, c->KP);
        ATJUP_CHECK_LAUNCH("bc_phi");
    }
    if (which & ATJUP_BC_SOLID) {
        if (c->n_solid > 0) {
            FieldList S{};
            add(S, t); add(S, p_stat); add(S, p_dyn);
            if (ph) { add_species(S); add_massflux(S, true); }
            c->launches++;
            solid_kernel<<<(c->n_solid + 127) / 128, 128, 0, c->stream>>>(c->solid_list, c->n_solid,
                                                                           S, u, v, w);
            if (P.mount_t_ambient && c->n_amb_rows > 0) {
                c->launches++;
                ambient_kernel<<<c->n_amb_rows, 32, 0, c->stream>>>(c->amb_rows, c->solid, t, P.jm,
                                                                   P.km, c->KP);
            }
        }
        if (ph) {
            SanArgs a{c->f[ATJUP_F_TKE], c->fn[ATJUP_F_TKE], c->f[ATJUP_F_DIS], c->fn[ATJUP_F_DIS],
                      c->f[ATJUP_F_NUE], c->f[ATJUP_F_PROD], c->f[ATJUP_F_TKE_SOURCE],
                      c->f[ATJUP_F_DIS_SOURCE], c->NP, 1000.0 / (P.u_0 * P.u_0),
                      1.0e5 / (P.u_0 * P.L_atm * 1.0e3)};
            c->launches++;
            sanitise_kernel<<<(unsigned)((c->NP + 255) / 256), 256, 0, c->stream>>>(a);
        }
        ATJUP_CHECK_LAUNCH("bc_solid");
    }
    return ATJUP_OK;
}

}  // namespace atjup
