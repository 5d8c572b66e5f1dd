// Poisson pressure solve, the reference's red-black form.
//
// Reference: PressureSolver<Planet>::run (PressureSolver.h:144-766) with
// cJupiterModel::prepareProjectionBoundaries (cJupiterModel.cpp:1842-1864).
// The operator relaxed per cell is  sum_{kept faces} num (p_nb - p) = src  with
// num1 = 1/dr^2, num2 = 1/(rm^2 dtheta^2), num3 = 1/(rm^2 s_j^2 dphi^2), s_j = max(sin, 0.55);
// faces into the obstacle are dropped for fluid cells (dp/dn = 0), solid cells keep the plain
// stencil. src = div(aux), one-sided at solid cells, clamped to |src| <= cap * den. After both
// colours the boundary values are folded from the interior: p[0] = 4/3 p[1] - 1/3 p[2] in r and
// theta, and the seam copy p[., ., km-1] = p[., ., 0].
//
// The source depends only on aux and the mask, which are fixed during a solve, so it is formed
// once per solve into ctx->src; each colour pass then reads p (7 points), the mask and src and
// writes half the cells. Within one colour every cell reads only cells of the other colour (the
// phi ring has an even number of meridians), so the parallel update equals the sequential one.
#include "ctx.cuh"

namespace atjup {
namespace {

constexpr double kC43 = 4.0 / 3.0, kC13 = 1.0 / 3.0;

struct PressConst {
    int im, jm, km, KP;
    double inv_dr2, inv_2dr, inv_2dthe, inv_2dphi, inv_dthe, inv_dphi;
    double cap;
    int press_wall;
};

// face weights and the face-dropping sum (PressureSolver.h:461-479)
__device__ __forceinline__ double gather(const double* __restrict__ p,
                                         const uint8_t* __restrict__ s, size_t c, size_t plane,
                                         size_t row, size_t ckp, size_t ckm, double n1, double n2,
                                         double n3, int press_wall, double* den_out) {
    double acc = 0.0, den;
    if (press_wall && !s[c]) {
        den = 0.0;
        if (!s[c + plane]) { acc += n1 * p[c + plane]; den += n1; }
        if (!s[c - plane]) { acc += n1 * p[c - plane]; den += n1; }
        if (!s[c + row]) { acc += n2 * p[c + row]; den += n2; }
        if (!s[c - row]) { acc += n2 * p[c - row]; den += n2; }
        if (!s[ckp]) { acc += n3 * p[ckp]; den += n3; }
        if (!s[ckm]) { acc += n3 * p[ckm]; den += n3; }
    } else {
        den = 2.0 * n1 + 2.0 * n2 + 2.0 * n3;
        acc = (p[c + plane] + p[c - plane]) * n1 + (p[c + row] + p[c - row]) * n2 +
              (p[ckp] + p[ckm]) * n3;
    }
    *den_out = den;
    return acc;
}

// Divergence source of one cell (PressureSolver.h:370-459), clamped (484-487).
// mask_out (optional): 1 where the clamp passes the divergence (finite, |div| <= cap den), else 0.
// mask_in (optional, the tangent-linear of the clamp about a base state): the divergence times
// mask_in, unclamped.
__global__ void source_kernel(const double* __restrict__ Su, const double* __restrict__ Sv,
                              const double* __restrict__ Sw, const uint8_t* __restrict__ s,
                              const GeoIJ* __restrict__ geo, double* __restrict__ src,
                              PressConst q, const uint8_t* __restrict__ mask_in,
                              uint8_t* __restrict__ mask_out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y + 1;
    const int i = blockIdx.z + 1;
    if (k > q.km - 2) return;
    const size_t row = q.KP, plane = (size_t)q.jm * row;
    const size_t c = (size_t)i * plane + (size_t)j * row + k;
    const int kw = (k == 0) ? q.km - 2 : k - 1;
    const int ke = (k == q.km - 2) ? 0 : k + 1;
    const size_t ckp = c - k + ke, ckm = c - k + kw;
    const GeoIJ& g = geo[i * q.jm + j];
    const double n1 = q.inv_dr2, n2 = g.num2, n3 = g.num3;
    // den of this cell (the stencil values are not needed here)
    double den;
    if (q.press_wall && !s[c]) {
        den = 0.0;
        if (!s[c + plane]) den += n1;
        if (!s[c - plane]) den += n1;
        if (!s[c + row]) den += n2;
        if (!s[c - row]) den += n2;
        if (!s[ckp]) den += n3;
        if (!s[ckm]) den += n3;
    } else {
        den = 2.0 * n1 + 2.0 * n2 + 2.0 * n3;
    }
    const int sld = s[c];
    const int sld_kp1 = s[ckp], sld_km1 = s[ckm];
    const int sld_kp2 = (k < q.km - 2) ? s[c + 2] : 0;
    const int sld_km2 = (k > 2) ? s[c - 2] : 0;
    double du_dr = 0.0, dv_dthe = 0.0, dw_dphi = 0.0;
    bool rf = false, tf = false, pf = false;
    if (i < q.im - 2 && sld && !s[c + plane]) {
        du_dr = (-3.0 * Su[c] + 4.0 * Su[c + plane] - Su[c + 2 * plane]) * q.inv_2dr;
        rf = true;
    }
    if (j > 2 && j < q.jm - 2) {
        const bool air_jp1 = !s[c + row], air_jm1 = !s[c - row];
        if (sld && air_jp1 && !s[c + 2 * row]) {
            dv_dthe = (-3.0 * Sv[c] + 4.0 * Sv[c + row] - Sv[c + 2 * row]) * q.inv_2dthe;
            tf = true;
        }
        if (sld && air_jm1 && !s[c - 2 * row]) {
            dv_dthe = -(-3.0 * Sv[c] + 4.0 * Sv[c - row] - Sv[c - 2 * row]) * q.inv_2dthe;
            tf = true;
        }
        if ((sld && air_jp1 && s[c + 2 * row]) || (j == q.jm - 2 && !sld && s[c + row])) {
            dv_dthe = (Sv[c + row] - Sv[c]) * q.inv_dthe;
            tf = true;
        }
        if ((sld && air_jm1 && s[c - 2 * row]) || (j == 1 && sld && air_jm1)) {
            dv_dthe = (Sv[c - row] - Sv[c]) * q.inv_dthe;
            tf = true;
        }
    }
    if (k > 2 && k < q.km - 2) {
        const bool air_kp1 = !sld_kp1, air_km1 = !sld_km1;
        if (sld && air_kp1 && !sld_kp2) {
            dw_dphi = (-3.0 * Sw[c] + 4.0 * Sw[c + 1] - Sw[c + 2]) * q.inv_2dphi;
            pf = true;
        }
        if (sld && air_km1 && !sld_km2) {
            dw_dphi = -(-3.0 * Sw[c] + 4.0 * Sw[c - 1] - Sw[c - 2]) * q.inv_2dphi;
            pf = true;
        }
        if ((sld && air_kp1 && sld_kp2) || (k == q.km - 2 && !sld && sld_kp1)) {
            dw_dphi = (Sw[c + 1] - Sw[c]) * q.inv_dphi;
            pf = true;
        }
        if ((sld && air_km1 && sld_km2) || (k == 1 && sld && air_km1)) {
            dw_dphi = (Sw[c - 1] - Sw[c]) * q.inv_dphi;
            pf = true;
        }
    }
    if (!rf) du_dr = (Su[c + plane] - Su[c - plane]) * q.inv_2dr;
    if (!tf) dv_dthe = (Sv[c + row] - Sv[c - row]) * q.inv_2dthe;
    if (!pf) dw_dphi = (Sw[ckp] - Sw[ckm]) * q.inv_2dphi;
    double div_src = du_dr * 1.0 + dv_dthe * g.inv_rm + dw_dphi * g.inv_rmsinthe;
    const double src_max = den * q.cap;
    if (mask_out) mask_out[c] = (isfinite(div_src) && fabs(div_src) <= src_max) ? 1 : 0;
    if (mask_in) { src[c] = mask_in[c] ? div_src : 0.0; return; }
    if (!isfinite(div_src)) div_src = 0.0;
    else if (div_src > src_max) div_src = src_max;
    else if (div_src < -src_max) div_src = -src_max;
    src[c] = div_src;
}

// One colour of the red-black sweep: thread x -> k = 2x + ((i + j + colour) & 1).
__global__ void sweep_kernel(double* __restrict__ p, const uint8_t* __restrict__ s,
                             const double* __restrict__ src, const GeoIJ* __restrict__ geo,
                             PressConst q, int colour, double omega) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y + 1;
    const int i = blockIdx.z + 1;
    const int k = 2 * x + ((i + j + colour) & 1);
    if (k > q.km - 2) return;
    const size_t row = q.KP, plane = (size_t)q.jm * row;
    const size_t c = (size_t)i * plane + (size_t)j * row + k;
    const int kw = (k == 0) ? q.km - 2 : k - 1;
    const int ke = (k == q.km - 2) ? 0 : k + 1;
    const GeoIJ& g = geo[i * q.jm + j];
    double den;
    const double acc = gather(p, s, c, plane, row, c - k + ke, c - k + kw, q.inv_dr2, g.num2,
                              g.num3, q.press_wall, &den);
    if (den <= 0.0) return;
    const double pgs = (acc - src[c]) / den;
    p[c] = (omega == 1.0) ? pgs : p[c] + omega * (pgs - p[c]);
}

__global__ void fold_r_kernel(double* __restrict__ p, int im, int jm, int km, int KP) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (k >= km) return;
    const size_t plane = (size_t)jm * KP, b = (size_t)j * KP + k;
    p[b] = kC43 * p[b + plane] - kC13 * p[b + 2 * plane];
    p[b + (im - 1) * plane] = kC43 * p[b + (im - 2) * plane] - kC13 * p[b + (im - 3) * plane];
}

__global__ void fold_t_kernel(double* __restrict__ p, int im, int jm, int km, int KP) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (k >= km) return;
    const size_t b = (size_t)i * jm * KP + k;
    p[b] = kC43 * p[b + KP] - kC13 * p[b + 2 * KP];
    p[b + (size_t)(jm - 1) * KP] =
        kC43 * p[b + (size_t)(jm - 2) * KP] - kC13 * p[b + (size_t)(jm - 3) * KP];
}

__global__ void seam_kernel(double* __restrict__ p, int im, int jm, int km, int KP) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (j >= jm) return;
    const size_t b = ((size_t)i * jm + j) * KP;
    p[b + km - 1] = p[b];
}

// cJupiterModel.cpp:1842-1864: aux at the radial walls before the divergence is taken.
__global__ void prepare_kernel(double* __restrict__ au, double* __restrict__ av,
                               double* __restrict__ aw, int im, int jm, int km, int KP,
                               int rigid) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y + 1;
    if (k > km - 2) return;
    const size_t plane = (size_t)jm * KP, b = (size_t)j * KP + k;
    const size_t t0 = b, t1 = b + plane, t2 = b + 2 * plane;
    const size_t e0 = b + (im - 1) * plane, e1 = b + (im - 2) * plane, e2 = b + (im - 3) * plane;
    if (rigid) {
        au[t0] = 0.0;
        au[e0] = 0.0;
    } else {
        au[t0] = kC43 * au[t1] - kC13 * au[t2];
        au[e0] = kC43 * au[e1] - kC13 * au[e2];
    }
    av[t0] = kC43 * av[t1] - kC13 * av[t2];
    av[e0] = kC43 * av[e1] - kC13 * av[e2];
    aw[t0] = kC43 * aw[t1] - kC13 * aw[t2];
    aw[e0] = kC43 * aw[e1] - kC13 * aw[e2];
}

PressConst make_const(const AtjupCtx* c) {
    const AtjupParams& P = c->P;
    PressConst q{};
    q.im = P.im; q.jm = P.jm; q.km = P.km; q.KP = c->KP;
    q.inv_dr2 = 1.0 / (P.dr * P.dr);
    q.inv_2dr = 1.0 / (2.0 * P.dr);
    q.inv_2dthe = 1.0 / (2.0 * P.dthe);
    q.inv_2dphi = 1.0 / (2.0 * P.dphi);
    q.inv_dthe = 1.0 / P.dthe;
    q.inv_dphi = 1.0 / P.dphi;
    q.cap = P.p_dyn_cap;
    q.press_wall = P.press_wall;
    return q;
}

}  // namespace

int launch_prepare_projection_ptr(AtjupCtx* c, double* au, double* av, double* aw) {
    const AtjupParams& P = c->P;
    dim3 grid((P.km - 1 + 127) / 128, P.jm - 2);
    c->launches++;
    prepare_kernel<<<grid, 128, 0, c->stream>>>(au, av, aw, P.im, P.jm, P.km, c->KP, P.rigid_lid);
    ATJUP_CHECK_LAUNCH("prepare_projection");
    return ATJUP_OK;
}

int launch_prepare_projection(AtjupCtx* c) {
    return launch_prepare_projection_ptr(c, c->f[ATJUP_F_AUX_U], c->f[ATJUP_F_AUX_V],
                                         c->f[ATJUP_F_AUX_W]);
}

int launch_pressure_source_ptr(AtjupCtx* c, const double* au, const double* av, const double* aw,
                               double* src, const uint8_t* mask_in, uint8_t* mask_out) {
    const AtjupParams& P = c->P;
    const PressConst q = make_const(c);
    dim3 grid((P.km - 1 + 127) / 128, P.jm - 2, P.im - 2);
    c->launches++;
    source_kernel<<<grid, 128, 0, c->stream>>>(au, av, aw, c->solid, c->geo, src, q, mask_in,
                                              mask_out);
    ATJUP_CHECK_LAUNCH("pressure_source");
    return ATJUP_OK;
}

int launch_pressure_source(AtjupCtx* c) {
    return launch_pressure_source_ptr(c, c->f[ATJUP_F_AUX_U], c->f[ATJUP_F_AUX_V],
                                      c->f[ATJUP_F_AUX_W], c->src, nullptr, nullptr);
}

int launch_pressure_sweep_ptr(AtjupCtx* c, double* p, const double* src, int colour, double omega) {
    const AtjupParams& P = c->P;
    const PressConst q = make_const(c);
    const int nx = (P.km - 1 + 1) / 2;
    dim3 grid((nx + 127) / 128, P.jm - 2, P.im - 2);
    c->launches++;
    sweep_kernel<<<grid, 128, 0, c->stream>>>(p, c->solid, src, c->geo, q, colour, omega);
    ATJUP_CHECK_LAUNCH("pressure_sweep");
    return ATJUP_OK;
}

int launch_pressure_sweep(AtjupCtx* c, int colour, double omega) {
    return launch_pressure_sweep_ptr(c, c->f[ATJUP_F_P_DYN], c->src, colour, omega);
}

int launch_pressure_fold(AtjupCtx* c, double* p) {
    const AtjupParams& P = c->P;
    c->launches++;
    fold_r_kernel<<<dim3((P.km + 127) / 128, P.jm), 128, 0, c->stream>>>(p, P.im, P.jm, P.km, c->KP);
    c->launches++;
    fold_t_kernel<<<dim3((P.km + 127) / 128, P.im), 128, 0, c->stream>>>(p, P.im, P.jm, P.km, c->KP);
    c->launches++;
    seam_kernel<<<dim3((P.jm + 127) / 128, P.im), 128, 0, c->stream>>>(p, P.im, P.jm, P.km, c->KP);
    ATJUP_CHECK_LAUNCH("pressure_fold");
    return ATJUP_OK;
}

}  // namespace atjup
