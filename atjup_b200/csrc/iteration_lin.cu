// Tangent-linear and adjoint of one whole dry iteration of cJupiterModel::Run's loop
// (cJupiterModel.cpp:1032-1381 with the dry knobs): on even iterations (and the first) the
// pressure pass (PressureSolver.h:144-766 with prepareProjectionBoundaries,
// cJupiterModel.cpp:1842-1864) and the mixture density (InitValues_Jup.cpp:717-740); every
// iteration RungeKuttaJup, the boundary passes (BC_Jup.h:185-658, BoundaryConditions.h:151-518),
// the in-loop 4th-order Shapiro filter of u, v, w (lib/Utils.cpp:334-453) and the column balance
// of v (InitValues_Jup.cpp:1500-1538). The reference has no derivative code.
//
// The linear state is nine fields: t, u, v, w, p_dyn, aux_u, aux_v, aux_w and rho_mix -- what one
// iteration reads from the previous one (aux is the projection source the next pressure pass
// reads; rho_mix is carried over odd iterations). Both directions linearise about the context's
// current state, taken as the iteration's input, and leave it as they found it: they run the
// forward pressure pass and mixture density on the context to reach the RK step's linearisation
// point, and put p_dyn, aux and rho_mix back at the end.
//
//   tangent-linear: the linear passes (the folds, sweeps, boundary passes, filter and balance) are
//     the forward kernels run on the perturbations; the source clamp passes the perturbation where
//     the base state's divergence is not clamped (its derivative), the mixture density and the RK
//     step are linearised (adjoint.cu).
//   adjoint: the passes in reverse, each the transpose of its forward kernel as a scatter or a
//     gather: the balance (column sums), the filter (gathers over each output's stencil), the
//     boundary passes (zonal sums, wall and pole folds, the seam, the solid cells and their
//     ambient rows), the RK step (adjoint.cu), the mixture density, and the pressure pass (per
//     sweep the folds, then the black and the red colour, each cell's value divided by its
//     weight sum scattered to its six neighbours and to the source; then the divergence source's
//     stencils with its one-sided forms at the obstacle; then the radial walls of aux).
#include "ctx.cuh"

namespace atjup {
namespace {

constexpr double kC43 = 4.0 / 3.0, kC13 = 1.0 / 3.0;

// the nine fields of the linear state
enum { LT = 0, LU, LV, LW, LP, LAU, LAV, LAW, LR, LN };

// ---------------------------------------------------------------------------------------------
// mixture density: rho = (p_stat + w p_dyn to_bar) 1e5 / (R_mix t t_ref), 0 where t t_ref <= 0 or
// the value is not finite
__global__ void mix_lin_kernel(const double* __restrict__ t, const double* __restrict__ ps,
                               const double* __restrict__ pd, double* __restrict__ dt,
                               double* __restrict__ dp, double* __restrict__ drho, size_t NP,
                               double t_ref, double pdyn_w, double to_bar, double R_mix,
                               int adjoint) {
    const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= NP) return;
    const double T = t[c] * t_ref;
    bool live = T > 0.0;
    double r = 0.0;
    if (live) {
        r = (ps[c] + pdyn_w * pd[c] * to_bar) * 1.0e5 / (R_mix * T);
        live = isfinite(r);
    }
    const double kp = live ? pdyn_w * to_bar * 1.0e5 / (R_mix * T) : 0.0;
    const double kt = live ? -r / t[c] : 0.0;
    if (!adjoint) {
        drho[c] = kt * dt[c] + kp * dp[c];
    } else {
        const double l = drho[c];
        dt[c] += kt * l;
        if (pdyn_w != 0.0) dp[c] += kp * l;
        drho[c] = 0.0;
    }
}

// ---------------------------------------------------------------------------------------------
// pressure pass transposes
struct PQ {
    int im, jm, km, KP;
    double inv_dr2, inv_2dr, inv_2dthe, inv_2dphi, inv_dthe, inv_dphi;
    int press_wall, rigid;
};

// the seam copy, then the theta folds, then the radial folds, transposed in that order
__global__ void seam_T_kernel(double* __restrict__ l, PQ q) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
    if (j >= q.jm) return;
    const size_t b = ((size_t)i * q.jm + j) * q.KP;
    l[b] += l[b + q.km - 1];
    l[b + q.km - 1] = 0.0;
}
__global__ void fold_t_T_kernel(double* __restrict__ l, PQ q) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
    if (k >= q.km) return;
    const size_t b = (size_t)i * q.jm * q.KP + k, R = q.KP;
    const double g0 = l[b], g1 = l[b + (size_t)(q.jm - 1) * R];
    l[b] = 0.0;
    l[b + (size_t)(q.jm - 1) * R] = 0.0;
    l[b + R] += kC43 * g0;
    l[b + 2 * R] -= kC13 * g0;
    l[b + (size_t)(q.jm - 2) * R] += kC43 * g1;
    l[b + (size_t)(q.jm - 3) * R] -= kC13 * g1;
}
__global__ void fold_r_T_kernel(double* __restrict__ l, PQ q) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (k >= q.km) return;
    const size_t plane = (size_t)q.jm * q.KP, b = (size_t)j * q.KP + k;
    const double g0 = l[b], g1 = l[b + (size_t)(q.im - 1) * plane];
    l[b] = 0.0;
    l[b + (size_t)(q.im - 1) * plane] = 0.0;
    l[b + plane] += kC43 * g0;
    l[b + 2 * plane] -= kC13 * g0;
    l[b + (size_t)(q.im - 2) * plane] += kC43 * g1;
    l[b + (size_t)(q.im - 3) * plane] -= kC13 * g1;
}

// One colour of the sweep, transposed: p_c = (sum_faces w p_nb - src_c) / den overwrote p_c, so
// its adjoint G = l_c / den goes to each kept neighbour (w G) and to the source (-G), and l_c is
// cleared. The colour's cells read only cells of the other colour, so the scatters never touch
// a cell of this colour.
__global__ void sweep_T_kernel(double* __restrict__ lp, double* __restrict__ ls,
                               const uint8_t* __restrict__ s, const GeoIJ* __restrict__ geo,
                               PQ q, int colour) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y + 1, i = blockIdx.z + 1;
    const int k = 2 * x + ((i + j + colour) & 1);
    if (k > q.km - 2) return;
    const size_t row = q.KP, plane = (size_t)q.jm * row;
    const size_t c = (size_t)i * plane + (size_t)j * row + k;
    const int kw = (k == 0) ? q.km - 2 : k - 1;
    const int ke = (k == q.km - 2) ? 0 : k + 1;
    const size_t ckp = c - k + ke, ckm = c - k + kw;
    const GeoIJ& g = geo[i * q.jm + j];
    const double n1 = q.inv_dr2, n2 = g.num2, n3 = g.num3;
    const bool drop = q.press_wall && !s[c];
    const bool kip = !drop || !s[c + plane], kim = !drop || !s[c - plane];
    const bool kjp = !drop || !s[c + row], kjm = !drop || !s[c - row];
    const bool kkp = !drop || !s[ckp], kkm = !drop || !s[ckm];
    const double den = (kip ? n1 : 0.0) + (kim ? n1 : 0.0) + (kjp ? n2 : 0.0) + (kjm ? n2 : 0.0) +
                       (kkp ? n3 : 0.0) + (kkm ? n3 : 0.0);
    if (!(den > 0.0)) return;
    const double G = lp[c] / den;
    lp[c] = 0.0;
    if (G == 0.0) return;
    ls[c] -= G;
    if (kip) atomicAdd(lp + c + plane, n1 * G);
    if (kim) atomicAdd(lp + c - plane, n1 * G);
    if (kjp) atomicAdd(lp + c + row, n2 * G);
    if (kjm) atomicAdd(lp + c - row, n2 * G);
    if (kkp) atomicAdd(lp + ckp, n3 * G);
    if (kkm) atomicAdd(lp + ckm, n3 * G);
}

// The divergence source transposed (the forward is pressure.cu's source_kernel, with its branch
// order: a later one-sided form overrides an earlier one): coef * l_src into the aux adjoints at
// the stencil's cells, where the base state's clamp passed the divergence (mask).
__global__ void source_T_kernel(const double* __restrict__ ls, const uint8_t* __restrict__ mask,
                                double* __restrict__ lu, double* __restrict__ lv,
                                double* __restrict__ lw, const uint8_t* __restrict__ s,
                                const GeoIJ* __restrict__ geo, PQ q) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y + 1, i = blockIdx.z + 1;
    if (k > q.km - 2) return;
    const size_t row = q.KP, plane = (size_t)q.jm * row;
    const size_t c = (size_t)i * plane + (size_t)j * row + k;
    const double L = ls[c];
    if (L == 0.0 || !mask[c]) return;
    const int kw = (k == 0) ? q.km - 2 : k - 1;
    const int ke = (k == q.km - 2) ? 0 : k + 1;
    const size_t ckp = c - k + ke, ckm = c - k + kw;
    const GeoIJ& g = geo[i * q.jm + j];
    const int sld = s[c];
    // radial
    if (i < q.im - 2 && sld && !s[c + plane]) {
        atomicAdd(lu + c, -3.0 * q.inv_2dr * L);
        atomicAdd(lu + c + plane, 4.0 * q.inv_2dr * L);
        atomicAdd(lu + c + 2 * plane, -q.inv_2dr * L);
    } else {
        atomicAdd(lu + c + plane, q.inv_2dr * L);
        atomicAdd(lu + c - plane, -q.inv_2dr * L);
    }
    // theta: the last case that holds decides
    const double Lt = L * g.inv_rm;
    int tcase = 0;
    if (j > 2 && j < q.jm - 2) {
        const bool air_jp1 = !s[c + row], air_jm1 = !s[c - row];
        if (sld && air_jp1 && !s[c + 2 * row]) tcase = 1;
        if (sld && air_jm1 && !s[c - 2 * row]) tcase = 2;
        if ((sld && air_jp1 && s[c + 2 * row]) || (j == q.jm - 2 && !sld && s[c + row])) tcase = 3;
        if ((sld && air_jm1 && s[c - 2 * row]) || (j == 1 && sld && air_jm1)) tcase = 4;
    }
    switch (tcase) {
    case 1:
        atomicAdd(lv + c, -3.0 * q.inv_2dthe * Lt);
        atomicAdd(lv + c + row, 4.0 * q.inv_2dthe * Lt);
        atomicAdd(lv + c + 2 * row, -q.inv_2dthe * Lt);
        break;
    case 2:
        atomicAdd(lv + c, 3.0 * q.inv_2dthe * Lt);
        atomicAdd(lv + c - row, -4.0 * q.inv_2dthe * Lt);
        atomicAdd(lv + c - 2 * row, q.inv_2dthe * Lt);
        break;
    case 3:
        atomicAdd(lv + c + row, q.inv_dthe * Lt);
        atomicAdd(lv + c, -q.inv_dthe * Lt);
        break;
    case 4:
        atomicAdd(lv + c - row, q.inv_dthe * Lt);
        atomicAdd(lv + c, -q.inv_dthe * Lt);
        break;
    default:
        atomicAdd(lv + c + row, q.inv_2dthe * Lt);
        atomicAdd(lv + c - row, -q.inv_2dthe * Lt);
    }
    // phi
    const double Lp = L * g.inv_rmsinthe;
    int pcase = 0;
    if (k > 2 && k < q.km - 2) {
        const int sld_kp1 = s[ckp], sld_km1 = s[ckm];
        const int sld_kp2 = (k < q.km - 2) ? s[c + 2] : 0;
        const int sld_km2 = (k > 2) ? s[c - 2] : 0;
        const bool air_kp1 = !sld_kp1, air_km1 = !sld_km1;
        if (sld && air_kp1 && !sld_kp2) pcase = 1;
        if (sld && air_km1 && !sld_km2) pcase = 2;
        if ((sld && air_kp1 && sld_kp2) || (k == q.km - 2 && !sld && sld_kp1)) pcase = 3;
        if ((sld && air_km1 && sld_km2) || (k == 1 && sld && air_km1)) pcase = 4;
    }
    switch (pcase) {
    case 1:
        atomicAdd(lw + c, -3.0 * q.inv_2dphi * Lp);
        atomicAdd(lw + c + 1, 4.0 * q.inv_2dphi * Lp);
        atomicAdd(lw + c + 2, -q.inv_2dphi * Lp);
        break;
    case 2:
        atomicAdd(lw + c, 3.0 * q.inv_2dphi * Lp);
        atomicAdd(lw + c - 1, -4.0 * q.inv_2dphi * Lp);
        atomicAdd(lw + c - 2, q.inv_2dphi * Lp);
        break;
    case 3:
        atomicAdd(lw + c + 1, q.inv_dphi * Lp);
        atomicAdd(lw + c, -q.inv_dphi * Lp);
        break;
    case 4:
        atomicAdd(lw + c - 1, q.inv_dphi * Lp);
        atomicAdd(lw + c, -q.inv_dphi * Lp);
        break;
    default:
        atomicAdd(lw + ckp, q.inv_2dphi * Lp);
        atomicAdd(lw + ckm, -q.inv_2dphi * Lp);
    }
}

// the radial walls of aux before the divergence (rigid lid: aux_u 0 there), transposed
__global__ void prepare_T_kernel(double* __restrict__ lu, double* __restrict__ lv,
                                 double* __restrict__ lw, PQ q) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y + 1;
    if (k > q.km - 2) return;
    const size_t plane = (size_t)q.jm * q.KP, b = (size_t)j * q.KP + k;
    const size_t t0 = b, t1 = b + plane, t2 = b + 2 * plane;
    const size_t e0 = b + (size_t)(q.im - 1) * plane, e1 = b + (size_t)(q.im - 2) * plane;
    const size_t e2 = b + (size_t)(q.im - 3) * plane;
    double* L[3] = {lu, lv, lw};
    for (int f = 0; f < 3; f++) {
        double* l = L[f];
        const double g0 = l[t0], g1 = l[e0];
        l[t0] = 0.0;
        l[e0] = 0.0;
        if (f == 0 && q.rigid) continue;
        l[t1] += kC43 * g0;
        l[t2] -= kC13 * g0;
        l[e1] += kC43 * g1;
        l[e2] -= kC13 * g1;
    }
}

// ---------------------------------------------------------------------------------------------
// boundary passes (the dry lists: t, u, v, w in the radius, theta and phi passes; t and p_dyn
// in the solid-cell pass; p_stat is a frozen input), transposed

// taper 3: the zonal means of v, w at levels im-3 and im-2 feed v, w at im-3 (1/3), im-2 (2/3)
// and im-1 (the im-2 mean): their adjoints per row, before the column pass clears im-1
__global__ void zsum_T_kernel(const double* __restrict__ lv, const double* __restrict__ lw,
                              double* __restrict__ zg, int im, int jm, int km, int KP) {
    const int j = blockIdx.x, f = blockIdx.y;
    const double* l = f ? lw : lv;
    const size_t plane = (size_t)jm * KP, b = (size_t)j * KP;
    double s3 = 0.0, s2 = 0.0, s1 = 0.0;
    for (int k = threadIdx.x; k < km; k += 32) {
        s3 += l[b + (size_t)(im - 3) * plane + k];
        s2 += l[b + (size_t)(im - 2) * plane + k];
        s1 += l[b + (size_t)(im - 1) * plane + k];
    }
    for (int o = 16; o > 0; o >>= 1) {
        s3 += __shfl_down_sync(0xffffffffu, s3, o);
        s2 += __shfl_down_sync(0xffffffffu, s2, o);
        s1 += __shfl_down_sync(0xffffffffu, s1, o);
    }
    if (threadIdx.x == 0) {
        zg[(size_t)(2 * f) * jm + j] = kC13 * s3;                   // d/d(mean at im-3)
        zg[(size_t)(2 * f + 1) * jm + j] = (2.0 / 3.0) * s2 + s1;   // d/d(mean at im-2)
    }
}

// one (j, k) column: the taper, the lid and the 2-point Neumann walls, transposed
__global__ void radius_T_kernel(double* __restrict__ lt, double* __restrict__ lu,
                                double* __restrict__ lv, double* __restrict__ lw, int im, int jm,
                                int km, int KP, int lid_u, int taper) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (k >= km) return;
    const size_t plane = (size_t)jm * KP, b = (size_t)j * KP + k;
    const size_t c1 = b + (size_t)(im - 1) * plane, c2 = b + (size_t)(im - 2) * plane;
    const size_t c3 = b + (size_t)(im - 3) * plane;
    if (taper != 0) {
        double* VW[2] = {lv, lw};
        for (int f = 0; f < 2; f++) {
            double* x = VW[f];
            x[c1] = 0.0;
            if (taper == 2) {
                const size_t c4 = b + (size_t)(im - 4) * plane;
                const double g2 = x[c2], g3 = x[c3];
                x[c2] = 0.0;
                x[c3] = 0.0;
                x[c4] += kC13 * g2 + (2.0 / 3.0) * g3;
            } else {
                x[c2] *= kC13;
                x[c3] *= 2.0 / 3.0;
            }
        }
    }
    if (lid_u) {
        lu[b] = 0.0;
        lu[c1] = 0.0;
    }
    double* L[4] = {lt, lu, lv, lw};
    for (int f = 0; f < 4; f++) {
        double* x = L[f];
        const double g0 = x[b], g1 = x[c1];
        x[b] = 0.0;
        x[c1] = 0.0;
        x[b + plane] += kC43 * g0;
        x[b + 2 * plane] -= kC13 * g0;
        x[c2] += kC43 * g1;
        x[c3] -= kC13 * g1;
    }
}

__global__ void zadd_T_kernel(double* __restrict__ lv, double* __restrict__ lw,
                              const double* __restrict__ zg, int im, int jm, int km, int KP) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (k >= km - 1) return;
    const size_t plane = (size_t)jm * KP, b = (size_t)j * KP + k;
    const double inv = 1.0 / (km - 1);
    lv[b + (size_t)(im - 3) * plane] += zg[j] * inv;
    lv[b + (size_t)(im - 2) * plane] += zg[jm + j] * inv;
    lw[b + (size_t)(im - 3) * plane] += zg[2 * jm + j] * inv;
    lw[b + (size_t)(im - 2) * plane] += zg[3 * jm + j] * inv;
}

// pole rows transposed: the pole copies, then the fill rows nfill .. 1
__global__ void theta_T_kernel(double* __restrict__ lt, double* __restrict__ lu,
                               double* __restrict__ lv, double* __restrict__ lw, int im, int jm,
                               int km, int KP, int nfill) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (k >= km) return;
    const size_t b = (size_t)i * jm * KP + k;
    auto at = [&](int jj) { return b + (size_t)jj * KP; };
    double* X[2] = {lt, lu};
    double* Z[2] = {lv, lw};
    for (int f = 0; f < 2; f++) {
        double* x = X[f];
        x[at(1)] += x[at(0)];
        x[at(0)] = 0.0;
        x[at(jm - 2)] += x[at(jm - 1)];
        x[at(jm - 1)] = 0.0;
        Z[f][at(0)] = 0.0;
        Z[f][at(jm - 1)] = 0.0;
    }
    if (nfill > 0) {
        const int jf = nfill + 1;
        for (int r = nfill; r >= 1; r--) {
            const double ramp = (double)r / (double)jf;
            for (int f = 0; f < 2; f++) {
                double* x = X[f];
                x[at(jf)] += x[at(r)];
                x[at(r)] = 0.0;
                x[at(jm - 1 - jf)] += x[at(jm - 1 - r)];
                x[at(jm - 1 - r)] = 0.0;
                double* z = Z[f];
                z[at(jf)] += ramp * z[at(r)];
                z[at(r)] = 0.0;
                z[at(jm - 1 - jf)] += ramp * z[at(jm - 1 - r)];
                z[at(jm - 1 - r)] = 0.0;
            }
        }
    }
}

__global__ void phi_T_kernel(double* __restrict__ lt, double* __restrict__ lu,
                             double* __restrict__ lv, double* __restrict__ lw, int jm, int km,
                             int KP) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (j >= jm) return;
    const size_t b = ((size_t)i * jm + j) * KP;
    double* L[4] = {lt, lu, lv, lw};
    for (int f = 0; f < 4; f++) {
        L[f][b] += L[f][b + km - 1];
        L[f][b + km - 1] = 0.0;
    }
}

// the ambient temperature of a row's solid cells (the mean of its fluid t), transposed
__global__ void ambient_T_kernel(const int32_t* __restrict__ rows, const uint8_t* __restrict__ s,
                                 double* __restrict__ lt, int km, int KP) {
    const int r = rows[blockIdx.x];
    const size_t b = (size_t)r * KP;
    double sum = 0.0;
    int n = 0;
    for (int k = threadIdx.x; k < km; k += 32) {
        if (s[b + k]) sum += lt[b + k];
        else n++;
    }
    for (int o = 16; o > 0; o >>= 1) {
        sum += __shfl_down_sync(0xffffffffu, sum, o);
        n += __shfl_down_sync(0xffffffffu, n, o);
    }
    sum = __shfl_sync(0xffffffffu, sum, 0);
    n = __shfl_sync(0xffffffffu, n, 0);
    if (n == 0) return;              // the forward leaves such a row alone
    const double share = sum / n;
    for (int k = threadIdx.x; k < km; k += 32) {
        if (s[b + k]) lt[b + k] = 0.0;
        else lt[b + k] += share;
    }
}

// the solid cells: velocities 0; t and p_dyn from their extrapolation pair (kind 1), else p_dyn
// 0 and t kept; the pairs are fluid cells, shared between solid cells (atomic adds)
__global__ void solid_T_kernel(const SolidCell* __restrict__ Ls, int n, double* __restrict__ lt,
                               double* __restrict__ lu, double* __restrict__ lv,
                               double* __restrict__ lw, double* __restrict__ lp) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const SolidCell sc = Ls[q];
    lu[sc.c] = 0.0;
    lv[sc.c] = 0.0;
    lw[sc.c] = 0.0;
    if (sc.kind == 1) {
        double* L[2] = {lt, lp};
        for (int f = 0; f < 2; f++) {
            const double g = L[f][sc.c];
            L[f][sc.c] = 0.0;
            if (g != 0.0) {
                atomicAdd(L[f] + sc.a, kC43 * g);
                atomicAdd(L[f] + sc.b, -kC13 * g);
            }
        }
    } else {
        lp[sc.c] = 0.0;
    }
}

// ---------------------------------------------------------------------------------------------
// 4th-order Shapiro pass (filters.cu), transposed as gathers: an input cell collects, from each
// output within two cells whose stencil reads it, the output's adjoint times the stencil weight.
// An output is filtered in 4th order (weights 1 - 6 c4, 4 c4, -c4), in 2nd order near walls and
// solids (1 - 2 c2, c2), or copied (1).
struct FQ {
    int im, jm, km, KP, use_topo;
    double c4, c2;
};
__device__ __forceinline__ int floor_at(const int32_t* topo, int use_topo, int j, int k, int km) {
    if (!use_topo) return 0;
    const int t = topo[(size_t)j * km + k];
    return t > 0 ? t : 0;
}
// weight of offset d (input = output + d) for an output of mode m (0 copy, 2, 4)
__device__ __forceinline__ double fweight(int m, int d, const FQ& q) {
    const int ad = d < 0 ? -d : d;
    if (m == 4) return ad == 0 ? 1.0 - 6.0 * q.c4 : (ad == 1 ? 4.0 * q.c4 : -q.c4);
    if (m == 2) return ad == 0 ? 1.0 - 2.0 * q.c2 : (ad == 1 ? q.c2 : 0.0);
    return ad == 0 ? 1.0 : 0.0;
}

__global__ void shapiro_i_T_kernel(const double* __restrict__ src, double* __restrict__ dst,
                                   const int32_t* __restrict__ topo, FQ q) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, i = blockIdx.z;
    if (k >= q.km) return;
    const size_t plane = (size_t)q.jm * q.KP;
    const size_t c = (size_t)i * plane + (size_t)j * q.KP + k;
    const int is = floor_at(topo, q.use_topo, j, k, q.km);
    double acc = 0.0;
    for (int d = -2; d <= 2; d++) {
        const int o = i - d;                 // the output reading this input at offset d
        if (o < 0 || o > q.im - 1) continue;
        int m = 0;
        if (o >= is && o - 1 >= is && o + 1 <= q.im - 1)
            m = (o - 2 >= is && o + 2 <= q.im - 1) ? 4 : 2;
        const double wgt = fweight(m, d, q);
        if (wgt != 0.0) acc += wgt * src[c - (ptrdiff_t)d * (ptrdiff_t)plane];
    }
    dst[c] = acc;
}

// the mode of the output at offset o (-2..2) from the nine flags f[0..8] "inside the fluid" at
// offsets -4..4: 4th order when its four neighbours are inside, 2nd order when only the nearest
// two are, else a copy
__device__ __forceinline__ int out_mode(const bool* f, int o) {
    const int x = o + 4;
    if (!(f[x] && f[x - 1] && f[x + 1])) return 0;
    return (f[x - 2] && f[x + 2]) ? 4 : 2;
}

__global__ void shapiro_j_T_kernel(const double* __restrict__ src, double* __restrict__ dst,
                                   const int32_t* __restrict__ topo, FQ q) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, i = blockIdx.z;
    if (k >= q.km) return;
    const size_t row = q.KP;
    const size_t c = ((size_t)i * q.jm + j) * row + k;
    bool f[9];
#pragma unroll
    for (int e = 0; e < 9; e++) {
        const int jj = j + e - 4;
        f[e] = jj >= 0 && jj <= q.jm - 1 && i >= floor_at(topo, q.use_topo, jj, k, q.km);
    }
    double acc = 0.0;
#pragma unroll
    for (int d = -2; d <= 2; d++) {
        const int o = j - d;                 // the output reading this input at offset d
        if (o < 0 || o > q.jm - 1) continue;
        const double wgt = fweight(out_mode(f, -d), d, q);
        if (wgt != 0.0) acc += wgt * src[c - (ptrdiff_t)d * (ptrdiff_t)row];
    }
    dst[c] = acc;
}

// the k pass on the ring of km-1 meridians; its output km-1 is the copy of output 0
__global__ void shapiro_k_T_kernel(const double* __restrict__ src, double* __restrict__ dst,
                                   const int32_t* __restrict__ topo, FQ q) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, i = blockIdx.z;
    if (k >= q.km) return;
    const size_t b = ((size_t)i * q.jm + j) * q.KP;
    if (k == q.km - 1) { dst[b + k] = 0.0; return; }   // the seam input is never read
    const int n = q.km - 1;
    auto ring = [n](int kk) { return kk < 0 ? kk + n : (kk >= n ? kk - n : kk); };
    bool f[9];
#pragma unroll
    for (int e = 0; e < 9; e++) f[e] = i >= floor_at(topo, q.use_topo, j, ring(k + e - 4), q.km);
    double acc = 0.0;
#pragma unroll
    for (int d = -2; d <= 2; d++) {
        const int o = ring(k - d);
        const double wgt = fweight(out_mode(f, -d), d, q);
        if (wgt != 0.0) acc += wgt * (src[b + o] + (o == 0 ? src[b + q.km - 1] : 0.0));
    }
    dst[b + k] = acc;
}

// ---------------------------------------------------------------------------------------------
// column balance of v, transposed. Forward: per open column (topo 0) of rows 1..jm-2 the
// trapezoid mean of r v over i; zonal: v -= (the row mean over open meridians k < km-1 of those
// means) in every open column of the row; else v -= the column's own mean in that column.
// The weight of v_i in a column mean is (0.5 dr r_i, doubled inside) / I0.
__device__ __forceinline__ double vbal_weight(const double* rad, int i, int im, double dr,
                                              double I0) {
    const double w = 0.5 * rad[i] * dr * ((i == 0 || i == im - 1) ? 1.0 : 2.0);
    return w / I0;
}
__device__ __forceinline__ double vbal_I0(const double* rad, int im, double dr) {
    double I0 = 0.0;
    for (int i = 0; i < im - 1; i++) I0 += 0.5 * (rad[i] + rad[i + 1]) * dr;
    return I0;
}

// zonal: per row, S = the sum of lv over its open columns (all i, all k) and the count of open
// meridians k < km-1
__global__ void vbal_row_T_kernel(const double* __restrict__ lv, const int32_t* __restrict__ topo,
                                  double* __restrict__ rs, int im, int jm, int km, int KP) {
    const int j = blockIdx.x + 1;
    const size_t plane = (size_t)jm * KP;
    double s = 0.0;
    int n = 0;
    for (int k = threadIdx.x; k < km; k += blockDim.x) {
        if (topo[(size_t)j * km + k] != 0) continue;
        if (k < km - 1) n++;
        for (int i = 0; i < im; i++) s += lv[(size_t)i * plane + (size_t)j * KP + k];
    }
    __shared__ double sh[8];
    __shared__ int shn[8];
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
        n += __shfl_down_sync(0xffffffffu, n, o);
    }
    if ((threadIdx.x & 31) == 0) { sh[threadIdx.x >> 5] = s; shn[threadIdx.x >> 5] = n; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        int tn = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) { t += sh[w]; tn += shn[w]; }
        rs[2 * j] = t;
        rs[2 * j + 1] = (double)tn;
    }
}

__global__ void vbal_sub_T_kernel(double* __restrict__ lv, const int32_t* __restrict__ topo,
                                  const double* __restrict__ rs, const double* __restrict__ rad,
                                  int im, int jm, int km, int KP, double dr, int zonal) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y + 1;
    if (k >= km || topo[(size_t)j * km + k] != 0) return;
    const size_t plane = (size_t)jm * KP, b = (size_t)j * KP + k;
    const double I0 = vbal_I0(rad, im, dr);
    double S;
    if (zonal) {
        if (k >= km - 1 || rs[2 * j + 1] <= 0.0) return;    // not among the meridians averaged
        S = rs[2 * j] / rs[2 * j + 1];
    } else {
        S = 0.0;
        for (int i = 0; i < im; i++) S += lv[b + (size_t)i * plane];
    }
    for (int i = 0; i < im; i++) lv[b + (size_t)i * plane] -= S * vbal_weight(rad, i, im, dr, I0);
}

// ---------------------------------------------------------------------------------------------
struct Scratch {
    double* base[5];    // the context's p_dyn, aux_u, aux_v, aux_w, rho_mix on entry
    double* src;        // the perturbed source, or the source's adjoint
    double* pstat;      // a stand-in p_stat for the tangent-linear boundary pass
    uint8_t* mask;      // the base state's clamp: 1 where the divergence passes
};

int scratch(AtjupCtx* c, Scratch& S) {
    if (!c->itlin) ATJUP_CUDA(cudaMalloc(&c->itlin, sizeof(double) * 8 * c->NP));
    double* p = c->itlin;
    for (int f = 0; f < 5; f++) { S.base[f] = p; p += c->NP; }
    S.src = p; p += c->NP;
    S.pstat = p; p += c->NP;
    S.mask = reinterpret_cast<uint8_t*>(p);
    return ATJUP_OK;
}

const int kBaseIds[5] = {ATJUP_F_P_DYN, ATJUP_F_AUX_U, ATJUP_F_AUX_V, ATJUP_F_AUX_W,
                         ATJUP_F_RHO_MIX};

int save_base(AtjupCtx* c, const Scratch& S, bool restore) {
    for (int f = 0; f < 5; f++) {
        double* live = c->f[kBaseIds[f]];
        ATJUP_CUDA(cudaMemcpyAsync(restore ? live : S.base[f], restore ? S.base[f] : live,
                                   sizeof(double) * c->NP, cudaMemcpyDeviceToDevice, c->stream));
    }
    return ATJUP_OK;
}

int check_supported(AtjupCtx* c, const char* who, int iter_n) {
    const AtjupParams& P = c->P;
    char msg[200];
    if (!c->grid_set) {
        snprintf(msg, sizeof(msg), "%s: atjup_gpu_set_grid was not called", who);
        set_error(msg);
        return ATJUP_ERR_ARG;
    }
    if (c->phys_on || P.has_nue || P.has_heating || c->micro_on) {
        snprintf(msg, sizeof(msg), "%s: the dry iteration only (no physics, nue or heating)", who);
        set_error(msg);
        return ATJUP_ERR_UNSUPPORTED;
    }
    if (P.press_sweeps < 1) {
        snprintf(msg, sizeof(msg), "%s: needs press_sweeps >= 1", who);
        set_error(msg);
        return ATJUP_ERR_UNSUPPORTED;
    }
    if (P.cone_proj_stride > 0 && iter_n % P.cone_proj_stride == 0) {
        snprintf(msg, sizeof(msg), "%s: the projection around the obstacle runs at this iteration "
                 "and has no linearisation here (cone_proj_stride)", who);
        set_error(msg);
        return ATJUP_ERR_UNSUPPORTED;
    }
    return ATJUP_OK;
}

// the forward pressure pass and mixture density on the context (the RK step's linearisation
// point), recording the clamp mask of the base source
int base_pressure_and_density(AtjupCtx* c, const Scratch& S) {
    const AtjupParams& P = c->P;
    int rc;
    if ((rc = launch_prepare_projection(c))) return rc;
    if ((rc = launch_pressure_source_ptr(c, c->f[ATJUP_F_AUX_U], c->f[ATJUP_F_AUX_V],
                                         c->f[ATJUP_F_AUX_W], c->src, nullptr, S.mask))) return rc;
    for (int s = 0; s < P.press_sweeps; s++) {
        if ((rc = launch_pressure_sweep(c, 0, 1.0))) return rc;
        if ((rc = launch_pressure_sweep(c, 1, 1.0))) return rc;
        if ((rc = launch_pressure_fold(c, c->f[ATJUP_F_P_DYN]))) return rc;
    }
    return launch_mixture_density(c);
}

PQ press_q(const AtjupCtx* c) {
    const AtjupParams& P = c->P;
    PQ q{};
    q.im = P.im; q.jm = P.jm; q.km = P.km; q.KP = c->KP;
    q.inv_dr2 = 1.0 / (P.dr * P.dr);
    q.inv_2dr = 1.0 / (2.0 * P.dr);
    q.inv_2dthe = 1.0 / (2.0 * P.dthe);
    q.inv_2dphi = 1.0 / (2.0 * P.dphi);
    q.inv_dthe = 1.0 / P.dthe;
    q.inv_dphi = 1.0 / P.dphi;
    q.press_wall = P.press_wall;
    q.rigid = P.rigid_lid;
    return q;
}

FQ filt_q(const AtjupCtx* c) {
    const AtjupParams& P = c->P;
    FQ q{};
    q.im = P.im; q.jm = P.jm; q.km = P.km; q.KP = c->KP;
    q.use_topo = 1;
    q.c4 = P.shapiro_strength / 16.0;
    q.c2 = P.shapiro_strength * 0.25;
    return q;
}

int mixture_lin(AtjupCtx* c, double* const x[LN], int adjoint) {
    const AtjupParams& P = c->P;
    const unsigned nb = (unsigned)((c->NP + 255) / 256);
    mix_lin_kernel<<<nb, 256, 0, c->stream>>>(
        c->f[ATJUP_F_T], c->f[ATJUP_F_P_STAT], c->f[ATJUP_F_P_DYN], x[LT], x[LP], x[LR], c->NP,
        P.t_ref, P.rho_pdyn ? 1.0 : 0.0, P.p_dyn_to_bar, P.R_mix, adjoint);
    c->launches++;
    ATJUP_CHECK_LAUNCH("iteration linear: mixture density");
    return ATJUP_OK;
}

int pressure_T(AtjupCtx* c, const Scratch& S, double* const a[LN]) {
    const AtjupParams& P = c->P;
    const PQ q = press_q(c);
    cudaStream_t st = c->stream;
    ATJUP_CUDA(cudaMemsetAsync(S.src, 0, sizeof(double) * c->NP, st));
    const int nx = (P.km - 1 + 1) / 2;
    const dim3 gsw((nx + 127) / 128, P.jm - 2, P.im - 2);
    for (int s = 0; s < P.press_sweeps; s++) {
        seam_T_kernel<<<dim3((P.jm + 127) / 128, P.im), 128, 0, st>>>(a[LP], q);
        fold_t_T_kernel<<<dim3((P.km + 127) / 128, P.im), 128, 0, st>>>(a[LP], q);
        fold_r_T_kernel<<<dim3((P.km + 127) / 128, P.jm), 128, 0, st>>>(a[LP], q);
        sweep_T_kernel<<<gsw, 128, 0, st>>>(a[LP], S.src, c->solid, c->geo, q, 1);
        sweep_T_kernel<<<gsw, 128, 0, st>>>(a[LP], S.src, c->solid, c->geo, q, 0);
        c->launches += 5;
    }
    source_T_kernel<<<dim3((P.km - 1 + 127) / 128, P.jm - 2, P.im - 2), 128, 0, st>>>(
        S.src, S.mask, a[LAU], a[LAV], a[LAW], c->solid, c->geo, q);
    prepare_T_kernel<<<dim3((P.km - 1 + 127) / 128, P.jm - 2), 128, 0, st>>>(a[LAU], a[LAV],
                                                                           a[LAW], q);
    c->launches += 2;
    ATJUP_CHECK_LAUNCH("iteration adjoint: pressure pass");
    return ATJUP_OK;
}

int pressure_tl(AtjupCtx* c, const Scratch& S, double* const d[LN]) {
    const AtjupParams& P = c->P;
    int rc;
    if ((rc = launch_prepare_projection_ptr(c, d[LAU], d[LAV], d[LAW]))) return rc;
    if ((rc = launch_pressure_source_ptr(c, d[LAU], d[LAV], d[LAW], S.src, S.mask, nullptr)))
        return rc;
    for (int s = 0; s < P.press_sweeps; s++) {
        if ((rc = launch_pressure_sweep_ptr(c, d[LP], S.src, 0, 1.0))) return rc;
        if ((rc = launch_pressure_sweep_ptr(c, d[LP], S.src, 1, 1.0))) return rc;
        if ((rc = launch_pressure_fold(c, d[LP]))) return rc;
    }
    return ATJUP_OK;
}

int bc_T(AtjupCtx* c, double* const a[LN]) {
    const AtjupParams& P = c->P;
    cudaStream_t st = c->stream;
    // solid cells (the ambient rows last in the forward, so first here)
    if (c->n_solid > 0) {
        if (P.mount_t_ambient && c->n_amb_rows > 0) {
            ambient_T_kernel<<<c->n_amb_rows, 32, 0, st>>>(c->amb_rows, c->solid, a[LT], P.km, c->KP);
            c->launches++;
        }
        solid_T_kernel<<<(c->n_solid + 127) / 128, 128, 0, st>>>(c->solid_list, c->n_solid, a[LT],
                                                                a[LU], a[LV], a[LW], a[LP]);
        c->launches++;
    }
    phi_T_kernel<<<dim3((P.jm + 127) / 128, P.im), 128, 0, st>>>(a[LT], a[LU], a[LV], a[LW], P.jm,
                                                                P.km, c->KP);
    theta_T_kernel<<<dim3((P.km + 127) / 128, P.im), 128, 0, st>>>(
        a[LT], a[LU], a[LV], a[LW], P.im, P.jm, P.km, c->KP, P.pole_fill_rows);
    c->launches += 2;
    if (P.top_taper == 3) {
        zsum_T_kernel<<<dim3(P.jm, 2), 32, 0, st>>>(a[LV], a[LW], c->zm, P.im, P.jm, P.km, c->KP);
        c->launches++;
    }
    radius_T_kernel<<<dim3((P.km + 127) / 128, P.jm), 128, 0, st>>>(
        a[LT], a[LU], a[LV], a[LW], P.im, P.jm, P.km, c->KP, P.lid_u, P.top_taper);
    c->launches++;
    if (P.top_taper == 3) {
        zadd_T_kernel<<<dim3((P.km - 1 + 127) / 128, P.jm), 128, 0, st>>>(a[LV], a[LW], c->zm,
                                                                          P.im, P.jm, P.km, c->KP);
        c->launches++;
    }
    ATJUP_CHECK_LAUNCH("iteration adjoint: boundary passes");
    return ATJUP_OK;
}

int shapiro_T(AtjupCtx* c, double* f) {
    const AtjupParams& P = c->P;
    const FQ q = filt_q(c);
    const dim3 grid((P.km + 127) / 128, P.jm, P.im);
    for (int p = 0; p < P.shapiro_inloop; p++) {
        shapiro_i_T_kernel<<<grid, 128, 0, c->stream>>>(f, c->tmp, c->topo, q);
        shapiro_j_T_kernel<<<grid, 128, 0, c->stream>>>(c->tmp, c->tmp2, c->topo, q);
        shapiro_k_T_kernel<<<grid, 128, 0, c->stream>>>(c->tmp2, f, c->topo, q);
        c->launches += 3;
    }
    ATJUP_CHECK_LAUNCH("iteration adjoint: Shapiro filter");
    return ATJUP_OK;
}

int balance_T(AtjupCtx* c, double* lv) {
    const AtjupParams& P = c->P;
    if (P.v_massbal_zonal) {
        vbal_row_T_kernel<<<P.jm - 2, 256, 0, c->stream>>>(lv, c->topo, c->dvc, P.im, P.jm, P.km,
                                                          c->KP);
        c->launches++;
    }
    vbal_sub_T_kernel<<<dim3((P.km + 127) / 128, P.jm - 2), 128, 0, c->stream>>>(
        lv, c->topo, c->dvc, c->rad, P.im, P.jm, P.km, c->KP, P.dr, P.v_massbal_zonal);
    c->launches++;
    ATJUP_CHECK_LAUNCH("iteration adjoint: column balance");
    return ATJUP_OK;
}

bool args_ok(double* const x[LN]) {
    if (!x) return false;
    for (int f = 0; f < LN; f++) if (!x[f]) return false;
    return true;
}

}  // namespace
}  // namespace atjup

using namespace atjup;

extern "C" {

int atjup_gpu_iteration_tlm(AtjupCtx* c, int32_t iter_n, int32_t first, int32_t parts,
                            double* const d[9]) {
    if (!c || !args_ok(d)) { set_error("iteration_tlm: null argument"); return ATJUP_ERR_ARG; }
    int rc = check_supported(c, "iteration_tlm", iter_n);
    if (rc) return rc;
    const AtjupParams& P = c->P;
    Scratch S;
    if ((rc = scratch(c, S))) return rc;
    const bool even = (iter_n % 2 == 0) || first;
    // only the even iterations' base pressure pass and mixture density change the context
    if (even && (rc = save_base(c, S, false))) return rc;
    if (even) {
        if ((rc = base_pressure_and_density(c, S))) return rc;
        // the perturbed pass reads the base clamp mask; the base state's p_dyn and aux are the
        // ones after its own pass (the RK step's linearisation point)
        if ((parts & ATJUP_LIN_PRESSURE) && (rc = pressure_tl(c, S, d))) return rc;
        if ((parts & ATJUP_LIN_MIXTURE) && (rc = mixture_lin(c, d, 0))) return rc;
    }
    if (parts & ATJUP_LIN_RK4) {
        double* d4[4] = {d[LT], d[LU], d[LV], d[LW]};
        double* daux[3] = {d[LAU], d[LAV], d[LAW]};
        if ((rc = rk4_tlm_ext(c, d4, d[LP], d[LR], daux))) return rc;
    }
    if ((parts & ATJUP_LIN_BC) &&
        (rc = launch_bc_ptrs(c, ATJUP_BC_ALL, d[LT], d[LU], d[LV], d[LW], d[LP], S.pstat, false)))
        return rc;
    if ((parts & ATJUP_LIN_SHAPIRO) && P.shapiro_inloop > 0) {
        for (int f = LU; f <= LW; f++)
            if ((rc = launch_shapiro(c, d[f], 4, P.shapiro_strength, P.shapiro_inloop, 1))) return rc;
    }
    if ((parts & ATJUP_LIN_BALANCE) && P.v_massbal_stride > 0 && iter_n % P.v_massbal_stride == 0) {
        if ((rc = launch_balance_v_buffers(d[LV], c->topo, c->rad, c->dvc, c->dvrow, P.im, P.jm,
                                           P.km, c->KP, P.dr, P.v_massbal_zonal, c->stream)))
            return rc;
    }
    return even ? save_base(c, S, true) : ATJUP_OK;
}

static int iteration_adjoint_impl(AtjupCtx* c, int32_t iter_n, int32_t first, int32_t parts,
                                  double* const a[9], const double* const* stages) {
    int rc = check_supported(c, "iteration_adjoint", iter_n);
    if (rc) return rc;
    const AtjupParams& P = c->P;
    Scratch S;
    if ((rc = scratch(c, S))) return rc;
    const bool even = (iter_n % 2 == 0) || first;
    if (even && (rc = save_base(c, S, false))) return rc;
    if (even && (rc = base_pressure_and_density(c, S))) return rc;
    if ((parts & ATJUP_LIN_BALANCE) && P.v_massbal_stride > 0 && iter_n % P.v_massbal_stride == 0 &&
        (rc = balance_T(c, a[LV])))
        return rc;
    if ((parts & ATJUP_LIN_SHAPIRO) && P.shapiro_inloop > 0) {
        for (int f = LU; f <= LW; f++)
            if ((rc = shapiro_T(c, a[f]))) return rc;
    }
    if ((parts & ATJUP_LIN_BC) && (rc = bc_T(c, a))) return rc;
    if (parts & ATJUP_LIN_RK4) {
        double* a4[4] = {a[LT], a[LU], a[LV], a[LW]};
        double* laux[3] = {a[LAU], a[LAV], a[LAW]};
        if ((rc = rk4_adjoint_ext(c, a4, a[LP], a[LR], laux, stages))) return rc;
    }
    if (even) {
        if ((parts & ATJUP_LIN_MIXTURE) && (rc = mixture_lin(c, a, 1))) return rc;
        if ((parts & ATJUP_LIN_PRESSURE) && (rc = pressure_T(c, S, a))) return rc;
    }
    return even ? save_base(c, S, true) : ATJUP_OK;
}

int atjup_gpu_iteration_adjoint(AtjupCtx* c, int32_t iter_n, int32_t first, int32_t parts,
                                double* const a[9]) {
    if (!c || !args_ok(a)) { set_error("iteration_adjoint: null argument"); return ATJUP_ERR_ARG; }
    return iteration_adjoint_impl(c, iter_n, first, parts, a, nullptr);
}

int atjup_gpu_iteration_adjoint_ckpt(AtjupCtx* c, int32_t iter_n, int32_t first, int32_t parts,
                                     double* const a[9], const double* const stages[12]) {
    if (!c || !args_ok(a) || !stages) { set_error("iteration_adjoint_ckpt: null argument"); return ATJUP_ERR_ARG; }
    for (int b = 0; b < 12; b++)
        if (!stages[b]) { set_error("iteration_adjoint_ckpt: null stage buffer"); return ATJUP_ERR_ARG; }
    return iteration_adjoint_impl(c, iter_n, first, parts, a, stages);
}

}  // extern "C"
