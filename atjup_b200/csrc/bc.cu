// Boundary passes of the dynamics fields after the RK step.
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

__global__ void radius_kernel(double* __restrict__ t, double* __restrict__ u,
                              double* __restrict__ v, double* __restrict__ w,
                              const double* __restrict__ zm, int im, int jm, int km, int KP,
                              int lid_u, int taper) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (k >= km) return;
    const size_t plane = (size_t)jm * KP, b = (size_t)j * KP + k;
    double* F[4] = {t, u, v, w};
#pragma unroll
    for (int f = 0; f < 4; f++) {
        double* x = F[f];
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
}

// Pole rows (BoundaryConditions.h:253-336): rows 1..nfill copy row nfill+1 for t, u and ramp
// r/(nfill+1) of it for v, w; the pole row copies row 1 (t, u) and is zero (v, w).
__global__ void theta_kernel(double* __restrict__ t, double* __restrict__ u,
                             double* __restrict__ v, double* __restrict__ w, int im, int jm,
                             int km, int KP, int nfill) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (k >= km) return;
    const size_t b = (size_t)i * jm * KP + k;
    auto at = [&](int jj) { return b + (size_t)jj * KP; };
    if (nfill > 0) {
        const int jf = nfill + 1;
        for (int r = 1; r <= nfill; r++) {
            const double ramp = (double)r / (double)jf;
            t[at(r)] = t[at(jf)];
            t[at(jm - 1 - r)] = t[at(jm - 1 - jf)];
            u[at(r)] = u[at(jf)];
            u[at(jm - 1 - r)] = u[at(jm - 1 - jf)];
            v[at(r)] = ramp * v[at(jf)];
            v[at(jm - 1 - r)] = ramp * v[at(jm - 1 - jf)];
            w[at(r)] = ramp * w[at(jf)];
            w[at(jm - 1 - r)] = ramp * w[at(jm - 1 - jf)];
        }
    }
    v[at(0)] = 0.0;
    v[at(jm - 1)] = 0.0;
    w[at(0)] = 0.0;
    w[at(jm - 1)] = 0.0;
    t[at(0)] = t[at(1)];
    t[at(jm - 1)] = t[at(jm - 2)];
    u[at(0)] = u[at(1)];
    u[at(jm - 1)] = u[at(jm - 2)];
}

__global__ void phi_kernel(double* __restrict__ t, double* __restrict__ u,
                           double* __restrict__ v, double* __restrict__ w, int jm, int km,
                           int KP) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (j >= jm) return;
    const size_t b = ((size_t)i * jm + j) * KP;
    t[b + km - 1] = t[b];
    u[b + km - 1] = u[b];
    v[b + km - 1] = v[b];
    w[b + km - 1] = w[b];
}

__global__ void solid_kernel(const SolidCell* __restrict__ L, int n, double* __restrict__ t,
                             double* __restrict__ u, double* __restrict__ v,
                             double* __restrict__ w, double* __restrict__ ps,
                             double* __restrict__ pd) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const SolidCell s = L[q];
    u[s.c] = 0.0;
    v[s.c] = 0.0;
    w[s.c] = 0.0;
    if (s.kind == 1) {
        t[s.c] = kC43 * t[s.a] - kC13 * t[s.b];
        ps[s.c] = kC43 * ps[s.a] - kC13 * ps[s.b];
        pd[s.c] = kC43 * pd[s.a] - kC13 * pd[s.b];
    } else {
        pd[s.c] = 0.0;
    }
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
    const AtjupParams& P = c->P;
    double* t = c->f[ATJUP_F_T];
    double* u = c->f[ATJUP_F_U];
    double* v = c->f[ATJUP_F_V];
    double* w = c->f[ATJUP_F_W];
    if (which & ATJUP_BC_RADIUS) {
        if (P.top_taper == 3) {
            c->launches++;
            zonal_mean_kernel<<<dim3(P.jm, 2), 32, 0, c->stream>>>(v, w, c->zm, P.im, P.jm, P.km, c->KP);
        }
        c->launches++;
        radius_kernel<<<dim3((P.km + 127) / 128, P.jm), 128, 0, c->stream>>>(
            t, u, v, w, c->zm, P.im, P.jm, P.km, c->KP, P.lid_u, P.top_taper);
        ATJUP_CHECK_LAUNCH("bc_radius");
    }
    if (which & ATJUP_BC_THETA) {
        c->launches++;
        theta_kernel<<<dim3((P.km + 127) / 128, P.im), 128, 0, c->stream>>>(
            t, u, v, w, P.im, P.jm, P.km, c->KP, P.pole_fill_rows);
        ATJUP_CHECK_LAUNCH("bc_theta");
    }
    if (which & ATJUP_BC_PHI) {
        c->launches++;
        phi_kernel<<<dim3((P.jm + 127) / 128, P.im), 128, 0, c->stream>>>(t, u, v, w, P.jm, P.km, c->KP);
        ATJUP_CHECK_LAUNCH("bc_phi");
    }
    if ((which & ATJUP_BC_SOLID) && c->n_solid > 0) {
        c->launches++;
        solid_kernel<<<(c->n_solid + 127) / 128, 128, 0, c->stream>>>(
            c->solid_list, c->n_solid, t, u, v, w, c->f[ATJUP_F_P_STAT], c->f[ATJUP_F_P_DYN]);
        if (P.mount_t_ambient && c->n_amb_rows > 0) {
            c->launches++;
            ambient_kernel<<<c->n_amb_rows, 32, 0, c->stream>>>(c->amb_rows, c->solid, t, P.jm,
                                                               P.km, c->KP);
        }
        ATJUP_CHECK_LAUNCH("bc_solid");
    }
    return ATJUP_OK;
}

}  // namespace atjup
