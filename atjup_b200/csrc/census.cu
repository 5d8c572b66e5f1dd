// NaN / Inf census of the prognostic fields (the reference's ATJUP_NANCHECK idea, FileIO_Jup.cpp:
// 326-373, as a device reduction that returns a count instead of trapping).
#include "ctx.cuh"

namespace atjup {
namespace {

__global__ void nonfinite_kernel(const double* __restrict__ a, const double* __restrict__ b,
                                 const double* __restrict__ c, const double* __restrict__ d,
                                 const double* __restrict__ e, size_t NP, int km, int KP,
                                 unsigned long long* __restrict__ count) {
    unsigned long long n = 0;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < NP;
         q += (size_t)gridDim.x * blockDim.x) {
        if ((int)(q % KP) >= km) continue;
        n += !isfinite(a[q]) + !isfinite(b[q]) + !isfinite(c[q]) + !isfinite(d[q]) + !isfinite(e[q]);
    }
    for (int o = 16; o > 0; o >>= 1) n += __shfl_down_sync(0xffffffffu, n, o);
    if ((threadIdx.x & 31) == 0 && n) atomicAdd(count, n);
}

__global__ void pad_kernel(const double* __restrict__ flat, double* __restrict__ padded,
                           size_t rows, int km, int KP, int dir) {
    const size_t n = rows * (size_t)km;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
         q += (size_t)gridDim.x * blockDim.x) {
        const size_t r = q / km, k = q - r * km;
        if (dir == 0) padded[r * KP + k] = flat[q];
        else const_cast<double*>(flat)[q] = padded[r * KP + k];
    }
}

}  // namespace

int launch_pad(AtjupCtx* c, const double* flat, double* padded) {
    c->launches++;
    pad_kernel<<<148 * 8, 256, 0, c->stream>>>(flat, padded, (size_t)c->P.im * c->P.jm, c->P.km,
                                               c->KP, 0);
    ATJUP_CHECK_LAUNCH("pad");
    return ATJUP_OK;
}

int launch_unpad(AtjupCtx* c, const double* padded, double* flat) {
    c->launches++;
    pad_kernel<<<148 * 8, 256, 0, c->stream>>>(flat, const_cast<double*>(padded),
                                               (size_t)c->P.im * c->P.jm, c->P.km, c->KP, 1);
    ATJUP_CHECK_LAUNCH("unpad");
    return ATJUP_OK;
}

int launch_nonfinite(AtjupCtx* c, unsigned long long* d_count) {
    c->launches++;
    nonfinite_kernel<<<148 * 4, 256, 0, c->stream>>>(c->f[ATJUP_F_T], c->f[ATJUP_F_U],
                                                    c->f[ATJUP_F_V], c->f[ATJUP_F_W],
                                                    c->f[ATJUP_F_P_DYN], c->NP, c->P.km, c->KP,
                                                    d_count);
    ATJUP_CHECK_LAUNCH("nonfinite");
    return ATJUP_OK;
}



}  // namespace atjup

extern "C" int atjup_gpu_set_solve_rhs(AtjupCtx* c, const double* host_b) {
    if (!c || !host_b) { atjup::set_error("set_solve_rhs: null argument"); return ATJUP_ERR_ARG; }
    const AtjupParams& P = c->P;
    if (!c->solve_b) {
        ATJUP_CUDA(cudaMalloc(&c->solve_b, sizeof(double) * c->NP));
        ATJUP_CUDA(cudaMemset(c->solve_b, 0, sizeof(double) * c->NP));
    }
    ATJUP_CUDA(cudaMemcpy2DAsync(c->solve_b, sizeof(double) * c->KP, host_b, sizeof(double) * P.km,
                                 sizeof(double) * P.km, (size_t)P.im * P.jm,
                                 cudaMemcpyHostToDevice, c->stream));
    ATJUP_CUDA(cudaStreamSynchronize(c->stream));
    return ATJUP_OK;
}
