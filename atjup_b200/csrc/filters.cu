// Shapiro filters and the column balance of v.
//
// Reference: JupiterUtils::damp_wiggles (lib/Utils.cpp:227-323, order 2) and damp_wiggles_ho
// (lib/Utils.cpp:334-453, order 4): direction-split passes k (periodic ring of km-1 meridians,
// k = km-1 written as the copy of k = 0), then j (clamped at the poles), then i (clamped at the
// fluid floor i_topography), each pass reading a full copy of the field. Here each pass is an
// out-of-place kernel that writes every cell (filtered, or copied where the reference skips),
// chained field -> tmp -> tmp2 -> field.
//
// cJupiterModel::balanceColumnV (InitValues_Jup.cpp:1500-1538): trapezoid column mean of r v
// over columns off the obstacle, then (zonal form) the row mean of those removed from every
// off-obstacle column of the row.
#include "ctx.cuh"

namespace atjup {
namespace {

struct FiltConst {
    int im, jm, km, KP, order, use_topo;
    double c4, c2;
};

__device__ __forceinline__ int floor_of(const int32_t* topo, int use_topo, int j, int k, int km) {
    if (!use_topo) return 0;
    const int t = topo[(size_t)j * km + k];
    return t > 0 ? t : 0;
}

__global__ void shapiro_k_kernel(const double* __restrict__ src, double* __restrict__ dst,
                                 const int32_t* __restrict__ topo, FiltConst q) {
    const int k_out = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, i = blockIdx.z;
    if (k_out >= q.km) return;
    const size_t b = ((size_t)i * q.jm + j) * q.KP;
    const int k = (k_out == q.km - 1) ? 0 : k_out;   // the seam copy takes k = 0's result
    const int n = q.km - 1;
    const double cc = src[b + k];
    double out = cc;
    auto inf = [&](int kk) { return i >= floor_of(topo, q.use_topo, j, kk, q.km); };
    if (inf(k)) {
        if (q.order == 4) {
            const int km1 = (k - 1 + n) % n, kp1 = (k + 1) % n;
            const int km2 = (k - 2 + n) % n, kp2 = (k + 2) % n;
            if (inf(km1) && inf(kp1)) {
                if (inf(km2) && inf(kp2)) {
                    const double d4 = src[b + kp2] - 4.0 * src[b + kp1] + 6.0 * cc -
                                      4.0 * src[b + km1] + src[b + km2];
                    out = cc - q.c4 * d4;
                } else {
                    out = cc + q.c2 * (src[b + km1] - 2.0 * cc + src[b + kp1]);
                }
            }
        } else {
            const int km1 = (k == 0) ? q.km - 2 : k - 1;
            const int kp1 = (k == q.km - 2) ? 0 : k + 1;
            const double vm = inf(km1) ? src[b + km1] : cc;
            const double vp = inf(kp1) ? src[b + kp1] : cc;
            out = cc + q.c2 * (vm - 2.0 * cc + vp);
        }
    }
    dst[b + k_out] = out;
}

__global__ void shapiro_j_kernel(const double* __restrict__ src, double* __restrict__ dst,
                                 const int32_t* __restrict__ topo, FiltConst q) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, i = blockIdx.z;
    if (k >= q.km) return;
    const size_t row = q.KP;
    const size_t c = ((size_t)i * q.jm + j) * row + k;
    const double cc = src[c];
    double out = cc;
    auto inf = [&](int jj) { return i >= floor_of(topo, q.use_topo, jj, k, q.km); };
    if (inf(j)) {
        if (q.order == 4) {
            const bool fm1 = (j - 1 >= 0) && inf(j - 1);
            const bool fp1 = (j + 1 <= q.jm - 1) && inf(j + 1);
            if (fm1 && fp1) {
                const bool fm2 = (j - 2 >= 0) && inf(j - 2);
                const bool fp2 = (j + 2 <= q.jm - 1) && inf(j + 2);
                if (fm2 && fp2) {
                    const double d4 = src[c + 2 * row] - 4.0 * src[c + row] + 6.0 * cc -
                                      4.0 * src[c - row] + src[c - 2 * row];
                    out = cc - q.c4 * d4;
                } else {
                    out = cc + q.c2 * (src[c - row] - 2.0 * cc + src[c + row]);
                }
            }
        } else {
            const int jm1 = j - 1 > 0 ? j - 1 : 0, jp1 = j + 1 < q.jm - 1 ? j + 1 : q.jm - 1;
            const size_t cm = c - (size_t)(j - jm1) * row, cp = c + (size_t)(jp1 - j) * row;
            const double vm = inf(jm1) ? src[cm] : cc;
            const double vp = inf(jp1) ? src[cp] : cc;
            out = cc + q.c2 * (vm - 2.0 * cc + vp);
        }
    }
    dst[c] = out;
}

__global__ void shapiro_i_kernel(const double* __restrict__ src, double* __restrict__ dst,
                                 const int32_t* __restrict__ topo, FiltConst q) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, i = blockIdx.z;
    if (k >= q.km) return;
    const size_t plane = (size_t)q.jm * q.KP;
    const size_t c = (size_t)i * plane + (size_t)j * q.KP + k;
    const int is = floor_of(topo, q.use_topo, j, k, q.km);
    const double cc = src[c];
    double out = cc;
    if (i >= is) {
        if (q.order == 4) {
            const bool fm1 = (i - 1 >= is), fp1 = (i + 1 <= q.im - 1);
            if (fm1 && fp1) {
                const bool fm2 = (i - 2 >= is), fp2 = (i + 2 <= q.im - 1);
                if (fm2 && fp2) {
                    const double d4 = src[c + 2 * plane] - 4.0 * src[c + plane] + 6.0 * cc -
                                      4.0 * src[c - plane] + src[c - 2 * plane];
                    out = cc - q.c4 * d4;
                } else {
                    out = cc + q.c2 * (src[c - plane] - 2.0 * cc + src[c + plane]);
                }
            }
        } else {
            const int im1 = i - 1 > is ? i - 1 : is, ip1 = i + 1 < q.im - 1 ? i + 1 : q.im - 1;
            out = cc + q.c2 * (src[c - (size_t)(i - im1) * plane] - 2.0 * cc +
                               src[c + (size_t)(ip1 - i) * plane]);
        }
    }
    dst[c] = out;
}

// balanceColumnV: column means (one thread per column, the reference's summation order)
__global__ void vcol_kernel(const double* __restrict__ v, const int32_t* __restrict__ topo,
                            const double* __restrict__ rad, double* __restrict__ dvc, int im,
                            int jm, int km, int KP, double dr) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y + 1;
    if (k >= km) return;
    const int i0 = topo[(size_t)j * km + k];
    if (i0 > 0) return;
    const size_t plane = (size_t)jm * KP, b = (size_t)j * KP + k;
    double I1 = 0.0, I0 = 0.0;
    for (int i = i0; i < im - 1; i++) {
        I1 += 0.5 * (rad[i] * v[b + i * plane] + rad[i + 1] * v[b + (i + 1) * plane]) * dr;
        I0 += 0.5 * (rad[i] + rad[i + 1]) * dr;
    }
    dvc[b] = I1 / I0;
}

// row mean over meridians k < km-1 of the off-obstacle column means (fixed-order reduction)
__global__ void vrow_kernel(const double* __restrict__ dvc, const int32_t* __restrict__ topo,
                            double* __restrict__ dvrow, int jm, int km, int KP) {
    const int j = blockIdx.x + 1;
    double s = 0.0;
    int n = 0;
    for (int k = threadIdx.x; k < km - 1; k += 32)
        if (topo[(size_t)j * km + k] == 0) { s += dvc[(size_t)j * KP + k]; n++; }
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
        n += __shfl_down_sync(0xffffffffu, n, o);
    }
    if (threadIdx.x == 0) dvrow[j] = (n > 0) ? s / n : 0.0;
}

__global__ void vsub_kernel(double* __restrict__ v, const int32_t* __restrict__ topo,
                            const double* __restrict__ dvrow, const double* __restrict__ dvc,
                            int jm, int km, int KP, int zonal) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y + 1;
    const int i = blockIdx.z;
    if (k >= km) return;
    const int i0 = topo[(size_t)j * km + k];
    if (i0 > 0) return;
    if (!zonal && i < i0) return;
    const size_t c = ((size_t)i * jm + j) * KP + k;
    v[c] -= zonal ? dvrow[j] : dvc[(size_t)j * KP + k];
}

}  // namespace

int launch_shapiro(AtjupCtx* c, double* f, int order, double strength, int passes, int use_topo) {
    const AtjupParams& P = c->P;
    FiltConst q{};
    q.im = P.im; q.jm = P.jm; q.km = P.km; q.KP = c->KP;
    q.order = order;
    q.use_topo = use_topo;
    q.c4 = strength / 16.0;
    q.c2 = strength * 0.25;
    double* tmp2 = c->tmp2;
    dim3 grid((P.km + 127) / 128, P.jm, P.im);
    for (int p = 0; p < passes; p++) {
        c->launches++;
        shapiro_k_kernel<<<grid, 128, 0, c->stream>>>(f, c->tmp, c->topo, q);
        c->launches++;
        shapiro_j_kernel<<<grid, 128, 0, c->stream>>>(c->tmp, tmp2, c->topo, q);
        c->launches++;
        shapiro_i_kernel<<<grid, 128, 0, c->stream>>>(tmp2, f, c->topo, q);
    }
    ATJUP_CHECK_LAUNCH("shapiro");
    return ATJUP_OK;
}

int launch_balance_v(AtjupCtx* c) {
    const AtjupParams& P = c->P;
    double* v = c->f[ATJUP_F_V];
    c->launches++;
    vcol_kernel<<<dim3((P.km + 127) / 128, P.jm - 2), 128, 0, c->stream>>>(
        v, c->topo, c->rad, c->dvc, P.im, P.jm, P.km, c->KP, P.dr);
    if (P.v_massbal_zonal) {
        c->launches++;
        vrow_kernel<<<P.jm - 2, 32, 0, c->stream>>>(c->dvc, c->topo, c->dvrow, P.jm, P.km, c->KP);
    }
    c->launches++;
    vsub_kernel<<<dim3((P.km + 127) / 128, P.jm - 2, P.im), 128, 0, c->stream>>>(
        v, c->topo, c->dvrow, c->dvc, P.jm, P.km, c->KP, P.v_massbal_zonal);
    ATJUP_CHECK_LAUNCH("balance_v");
    return ATJUP_OK;
}

// The column balance of v on caller-supplied buffers (the no-allocation entry point in
// noalloc.cu supplies its file-scope scratch): v [im][jm][pitch], topo [jm * km], rad [im],
// dvc [jm * pitch], dvrow [jm].
int launch_balance_v_buffers(double* v, const int32_t* topo, const double* rad, double* dvc,
                             double* dvrow, int im, int jm, int km, int pitch, double dr,
                             int zonal, cudaStream_t st) {
    vcol_kernel<<<dim3((km + 127) / 128, jm - 2), 128, 0, st>>>(v, topo, rad, dvc, im, jm, km, pitch, dr);
    if (zonal) vrow_kernel<<<jm - 2, 32, 0, st>>>(dvc, topo, dvrow, jm, km, pitch);
    vsub_kernel<<<dim3((km + 127) / 128, jm - 2, im), 128, 0, st>>>(v, topo, dvrow, dvc, jm, km, pitch, zonal);
    ATJUP_CHECK_LAUNCH("balance_v_buffers");
    return ATJUP_OK;
}

}  // namespace atjup
