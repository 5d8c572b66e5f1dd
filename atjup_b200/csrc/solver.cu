// Residual-controlled solve of the reference's pressure operator (ATJUP_SOLVE_RESIDUAL).
//
// The reference relaxes  A p = src  with red-black Gauss-Seidel sweeps and never forms a residual
// (PressureSolver.h:318-491). A is the 7-point metric Laplacian over the interior fluid cells
// (i = 1..im-2, j = 1..jm-2, k on the ring of km-1 meridians), faces into the obstacle dropped,
// boundary neighbours read through the 2-point Neumann folds p0 = 4/3 p1 - 1/3 p2 the sweep
// applies after every pass (PressureSolver.h:718-746). Its fixed point is what this solver
// computes, to a stated relative residual ||src - A p|| / ||src||.
//
// A is not symmetric (the folds), but D A is, for D = diag(y), y(i,j,k) = a_i d_j with
// a, d = (3/2, 1, ..., 1, 3/2): y is A's left null vector, so the right-hand side is first made
// compatible by removing its y-component, b <- b - (y.b / y.1) 1. The solve is preconditioned CG
// on -D A with a two-level SPD preconditioner built for this operator's 1e5 anisotropy
// (1/dr^2 = 1600 against 1/(r^2 dtheta^2) ~ 0.013):
//   - radial lines: each (j, k) column's tridiagonal part of A (all horizontal faces on the
//     diagonal) solved exactly -- this removes the radial stiffness;
//   - column modes: the column-constant fields, whose operator V^T (-D A) V is the 2-D horizontal
//     Laplacian d_j (S2 L_theta + S3_j L_phi) of the obstacle-free column sums; solved exactly by a
//     discrete Fourier transform over the meridian ring and one tridiagonal system in theta per
//     wavenumber (the reference's PRESS_BAROTROPIC idea, PressureSolver.h:49-67, 573-708, used
//     here as a preconditioner, so the obstacle need not be obstacle-free).
// Mixed precision: the Krylov vectors, the residual b - A p and the update of p stay FP64; the
// preconditioner (the radial line solves and the column-mode solve) runs in FP32.
#include "ctx.cuh"

#include <cmath>
#include <cstdio>
#include <type_traits>
#include <vector>

namespace atjup {
namespace {

constexpr int RB = 256;          // threads per reduction block
constexpr int NRED = 592;        // reduction blocks (4 per SM)
constexpr double kC43 = 4.0 / 3.0, kC13 = 1.0 / 3.0;

template <typename T>
struct Vecs {
    T *b = nullptr, *p = nullptr, *r = nullptr, *z = nullptr, *d = nullptr, *q = nullptr;
    T *la = nullptr, *lc = nullptr, *lm = nullptr;   // line factors (lower, modified upper, 1/pivot)
    T *g = nullptr;                                  // column sums [jm * km]
    T *gh = nullptr;                                 // spectra [2 * (NM+1) * J]
    T *cs = nullptr, *sn = nullptr;                  // DFT tables [(NM+1) * N]
    T *ta = nullptr, *tcp = nullptr, *tm = nullptr;  // theta tridiagonal factors [(NM+1) * J]
    T *S3d = nullptr, *dj = nullptr;                 // per-row S3_j, d_j
};

struct Solver {
    int NM = 0, N = 0, J = 0;
    Vecs<double> v64;
    Vecs<float> v32;
    double* part = nullptr;       // [NRED * 2] reduction partials
    double* scal = nullptr;       // device scalars: 0 rho, 1 alpha, 2 beta, 3 rr, 4 dq, 5 yb, 6 y1, 7 bb
    double* hs = nullptr;         // pinned host mirror of scal
    double* yw = nullptr;         // y on fluid interior cells, 0 elsewhere
    bool ready = false;
};

// ---------------------------------------------------------------------------------------------
struct OpC {
    int im, jm, km, KP;
    double n1;
};

__device__ __forceinline__ bool interior(int i, int j, int k, const OpC& q) {
    return i >= 1 && i <= q.im - 2 && j >= 1 && j <= q.jm - 2 && k <= q.km - 2;
}

// (A x)(c) on fluid interior cells; 0 elsewhere. Also accumulates sum y d (A d) when w != null.
template <typename T>
__global__ void __launch_bounds__(RB)
apply_kernel(const T* __restrict__ x, T* __restrict__ y, const uint8_t* __restrict__ s,
             const GeoIJ* __restrict__ geo, const double* __restrict__ yw, OpC q,
             double* __restrict__ part) {
    const size_t plane = (size_t)q.jm * q.KP, row = q.KP;
    const size_t NP = (size_t)q.im * plane;
    double acc_dot = 0.0;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < NP;
         c += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(c % row);
        const int j = (int)((c / row) % q.jm);
        const int i = (int)(c / plane);
        T out = 0;
        if (interior(i, j, k, q) && !s[c]) {
            const GeoIJ& g = geo[i * q.jm + j];
            const T n1 = (T)q.n1, n2 = (T)g.num2, n3 = (T)g.num3;
            const T xc = x[c];
            const int kw = (k == 0) ? q.km - 2 : k - 1;
            const int ke = (k == q.km - 2) ? 0 : k + 1;
            // a sum of differences (no cancellation of a large smooth x); a folded boundary face
            // contributes num (1/3)(x_c - x_inward)
            const T t13 = (T)kC13;
            T acc = 0;
            if (!s[c + plane])
                acc += (i + 1 == q.im - 1) ? n1 * t13 * (xc - x[c - plane]) : n1 * (x[c + plane] - xc);
            if (!s[c - plane])
                acc += (i - 1 == 0) ? n1 * t13 * (xc - x[c + plane]) : n1 * (x[c - plane] - xc);
            if (!s[c + row])
                acc += (j + 1 == q.jm - 1) ? n2 * t13 * (xc - x[c - row]) : n2 * (x[c + row] - xc);
            if (!s[c - row])
                acc += (j - 1 == 0) ? n2 * t13 * (xc - x[c + row]) : n2 * (x[c - row] - xc);
            if (!s[c - k + ke]) acc += n3 * (x[c - k + ke] - xc);
            if (!s[c - k + kw]) acc += n3 * (x[c - k + kw] - xc);
            out = acc;
            if (part) acc_dot += yw[c] * (double)xc * (double)out;
        }
        y[c] = out;
    }
    if (part) {
        __shared__ double sh[RB / 32];
        for (int o = 16; o > 0; o >>= 1) acc_dot += __shfl_down_sync(0xffffffffu, acc_dot, o);
        if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc_dot;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int w = 0; w < RB / 32; w++) t += sh[w];
            part[blockIdx.x] = t;
        }
    }
}

// generic weighted dot partials: sum w a b (w may be null = 1)
template <typename Ta, typename Tb>
__global__ void __launch_bounds__(RB)
dot_kernel(const Ta* __restrict__ a, const Tb* __restrict__ b, const double* __restrict__ w,
           size_t n, double* __restrict__ part) {
    double acc = 0.0;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (size_t)gridDim.x * blockDim.x)
        acc += (w ? w[c] : 1.0) * (double)a[c] * (double)b[c];
    __shared__ double sh[RB / 32];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < RB / 32; q++) t += sh[q];
        part[blockIdx.x] = t;
    }
}

// Sum the partials in a fixed order into scal[slot]; op: 0 store, 1 alpha = rho / sum,
// 2 beta = sum / rho and rho = sum.
__global__ void finalize_kernel(const double* __restrict__ part, int n, double* __restrict__ scal,
                                int slot, int op) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double t = 0.0;
    for (int q = 0; q < n; q++) t += part[q];
    scal[slot] = t;
    if (op == 1) scal[1] = (t != 0.0) ? scal[0] / t : 0.0;
    if (op == 2) { scal[2] = (scal[0] != 0.0) ? t / scal[0] : 0.0; scal[0] = t; }
}

// p += alpha d; r -= alpha q; partial sums of r^2
template <typename T>
__global__ void __launch_bounds__(RB)
update_kernel(T* __restrict__ p, T* __restrict__ r, const T* __restrict__ d, const T* __restrict__ q,
              const double* __restrict__ scal, size_t n, double* __restrict__ part) {
    const T alpha = (T)scal[1];
    double acc = 0.0;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (size_t)gridDim.x * blockDim.x) {
        p[c] += alpha * d[c];
        const T rn = r[c] - alpha * q[c];
        r[c] = rn;
        acc += (double)rn * (double)rn;
    }
    __shared__ double sh[RB / 32];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < RB / 32; w++) t += sh[w];
        part[blockIdx.x] = t;
    }
}

template <typename T>
__global__ void direction_kernel(double* __restrict__ d, const T* __restrict__ z,
                                 const double* __restrict__ scal, size_t n, int first) {
    const double beta = first ? 0.0 : scal[2];
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (size_t)gridDim.x * blockDim.x)
        d[c] = first ? (double)z[c] : (double)z[c] + beta * d[c];
}

// Radial line solve A_line z = r per (j, k) column, and the column sum g = sum_i y r.
template <typename T>
__global__ void line_kernel(const double* __restrict__ r, T* __restrict__ z, const T* __restrict__ la,
                            const T* __restrict__ lc, const T* __restrict__ lm,
                            const double* __restrict__ yw, T* __restrict__ g, OpC q) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y + 1;
    if (k > q.km - 2) return;
    const size_t plane = (size_t)q.jm * q.KP, b = (size_t)j * q.KP + k;
    T prev = 0;
    double gs = 0.0;
    for (int i = 1; i <= q.im - 2; i++) {
        const size_t c = b + (size_t)i * plane;
        const T m = lm[c];
        if (m == (T)0) { prev = 0; continue; }           // not a fluid interior cell
        gs += yw[c] * r[c];
        prev = ((T)r[c] - la[c] * prev) * m;
        z[c] = prev;
    }
    T next = 0;
    for (int i = q.im - 2; i >= 1; i--) {
        const size_t c = b + (size_t)i * plane;
        if (lm[c] == (T)0) { next = 0; continue; }
        next = z[c] - lc[c] * next;
        z[c] = next;
    }
    g[(size_t)j * q.km + k] = (T)gs;
}

// forward real DFT of g over the ring: gh[0][m][jj] = sum_k g cos, gh[1][m][jj] = sum_k g sin
template <typename T>
__global__ void dft_fwd_kernel(const T* __restrict__ g, const T* __restrict__ cs,
                               const T* __restrict__ sn, T* __restrict__ gh, int N, int NM, int J,
                               int km) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    const int jj = blockIdx.y;
    if (m > NM) return;
    const T* gr = g + (size_t)(jj + 1) * km;
    const T* cr = cs + (size_t)m * N;
    const T* sr = sn + (size_t)m * N;
    double a = 0.0, b = 0.0;
    for (int k = 0; k < N; k++) { a += (double)gr[k] * (double)cr[k]; b += (double)gr[k] * (double)sr[k]; }
    gh[(size_t)m * J + jj] = (T)a;
    gh[(size_t)(NM + 1) * J + (size_t)m * J + jj] = (T)b;
}

// per wavenumber and part: d_j (S2 L_theta - S3_j lam_m) e = g_hat, folded ends; factors
// precomputed (mode 0: row 1 pinned).
template <typename T>
__global__ void theta_solve_kernel(T* __restrict__ gh, const T* __restrict__ ta,
                                   const T* __restrict__ tcp, const T* __restrict__ tm,
                                   const T* __restrict__ dj, int NM, int J, int N) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    const int part = blockIdx.y;
    if (m > NM) return;
    if (part == 1 && (m == 0 || 2 * m == N)) {
        T* e = gh + (size_t)(NM + 1) * J + (size_t)m * J;
        for (int jj = 0; jj < J; jj++) e[jj] = 0;
        return;
    }
    T* e = gh + (size_t)part * (NM + 1) * J + (size_t)m * J;
    T mean0 = 0;
    if (m == 0) {
        // the zonal-mean problem is singular (constant null vector): drop the incompatible part
        // of its right-hand side, sum_j ghat_j = 0, before pinning the gauge
        double sg = 0.0;
        for (int jj = 0; jj < J; jj++) sg += (double)e[jj];
        mean0 = (T)(sg / J);
    }
    const T* a = ta + (size_t)m * J;
    const T* cp = tcp + (size_t)m * J;
    const T* mm = tm + (size_t)m * J;
    T prev = 0;
    for (int jj = 0; jj < J; jj++) {
        T rhs = (e[jj] - mean0) / dj[jj + 1];
        if (m == 0 && jj == 0) rhs = 0;                   // pinned gauge row
        prev = (rhs - a[jj] * prev) * mm[jj];
        e[jj] = prev;
    }
    T next = 0;
    for (int jj = J - 1; jj >= 0; jj--) {
        next = e[jj] - cp[jj] * next;
        e[jj] = next;
    }
}

// inverse DFT, add the column correction to z, and partial sums of y r z
template <typename T>
__global__ void __launch_bounds__(128)
dft_inv_kernel(const T* __restrict__ gh, const T* __restrict__ cs, const T* __restrict__ sn,
               T* __restrict__ z, const double* __restrict__ r, const double* __restrict__ yw,
               const T* __restrict__ lm, OpC q, int N, int NM, int J, double* __restrict__ part) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int jj = blockIdx.y;
    double acc = 0.0;
    if (k < N) {
        double e = 0.0;
        for (int m = 0; m <= NM; m++) {
            const double w = (m == 0 || 2 * m == N) ? 1.0 : 2.0;
            const double c = (double)cs[(size_t)m * N + k];
            const double s = (double)sn[(size_t)m * N + k];
            e += w * ((double)gh[(size_t)m * J + jj] * c +
                      ((m == 0 || 2 * m == N) ? 0.0 : (double)gh[(size_t)(NM + 1) * J + (size_t)m * J + jj] * s));
        }
        e /= N;
        const size_t plane = (size_t)q.jm * q.KP, b = (size_t)(jj + 1) * q.KP + k;
        for (int i = 1; i <= q.im - 2; i++) {
            const size_t c = b + (size_t)i * plane;
            if (lm[c] == (T)0) continue;
            const T zn = z[c] + (T)e;
            z[c] = zn;
            acc += yw[c] * r[c] * (double)zn;
        }
    }
    __shared__ double sh[4];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) part[blockIdx.y * gridDim.x + blockIdx.x] = sh[0] + sh[1] + sh[2] + sh[3];
}

// p64 += e64
__global__ void add_kernel(double* __restrict__ p, const double* __restrict__ e, size_t n) {
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (size_t)gridDim.x * blockDim.x)
        p[c] += e[c];
}

// r = b - A p in FP64 on fluid interior cells, with partial sums of r^2 and of v^2, v = |A| |p|:
// eps * ||v|| is the rounding floor of the residual of an FP64 p (one ulp of p moves it that much).
__global__ void __launch_bounds__(RB)
residual_kernel(const double* __restrict__ b, const double* __restrict__ x, double* __restrict__ r,
                const uint8_t* __restrict__ s, const GeoIJ* __restrict__ geo,
                const double* __restrict__ yw, OpC q, double* __restrict__ part) {
    const size_t plane = (size_t)q.jm * q.KP, row = q.KP;
    const size_t NP = (size_t)q.im * plane;
    double acc_r = 0.0, acc_v = 0.0;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < NP;
         c += (size_t)gridDim.x * blockDim.x) {
        double out = 0.0;
        if (yw[c] > 0.0) {
            const int k = (int)(c % row);
            const int j = (int)((c / row) % q.jm);
            const int i = (int)(c / plane);
            const GeoIJ& g = geo[i * q.jm + j];
            const double n1 = q.n1, n2 = g.num2, n3 = g.num3, xc = x[c];
            const int kw = (k == 0) ? q.km - 2 : k - 1;
            const int ke = (k == q.km - 2) ? 0 : k + 1;
            double t[6] = {0, 0, 0, 0, 0, 0};
            if (!s[c + plane]) t[0] = (i + 1 == q.im - 1) ? n1 * kC13 * (xc - x[c - plane]) : n1 * (x[c + plane] - xc);
            if (!s[c - plane]) t[1] = (i - 1 == 0) ? n1 * kC13 * (xc - x[c + plane]) : n1 * (x[c - plane] - xc);
            if (!s[c + row]) t[2] = (j + 1 == q.jm - 1) ? n2 * kC13 * (xc - x[c - row]) : n2 * (x[c + row] - xc);
            if (!s[c - row]) t[3] = (j - 1 == 0) ? n2 * kC13 * (xc - x[c + row]) : n2 * (x[c - row] - xc);
            if (!s[c - k + ke]) t[4] = n3 * (x[c - k + ke] - xc);
            if (!s[c - k + kw]) t[5] = n3 * (x[c - k + kw] - xc);
            const double ax = ((t[0] + t[1]) + (t[2] + t[3])) + (t[4] + t[5]);
            // (|A| |x|)_c: the size of the terms whose rounding bounds the residual of an FP64 x
            double den = 0.0, nb = 0.0;
            if (!s[c + plane]) { const double w = (i + 1 == q.im - 1) ? n1 * kC13 : n1; den += w; nb += w * fabs((i + 1 == q.im - 1) ? x[c - plane] : x[c + plane]); }
            if (!s[c - plane]) { const double w = (i - 1 == 0) ? n1 * kC13 : n1; den += w; nb += w * fabs((i - 1 == 0) ? x[c + plane] : x[c - plane]); }
            if (!s[c + row]) { const double w = (j + 1 == q.jm - 1) ? n2 * kC13 : n2; den += w; nb += w * fabs((j + 1 == q.jm - 1) ? x[c - row] : x[c + row]); }
            if (!s[c - row]) { const double w = (j - 1 == 0) ? n2 * kC13 : n2; den += w; nb += w * fabs((j - 1 == 0) ? x[c + row] : x[c - row]); }
            if (!s[c - k + ke]) { den += n3; nb += n3 * fabs(x[c - k + ke]); }
            if (!s[c - k + kw]) { den += n3; nb += n3 * fabs(x[c - k + kw]); }
            const double v = den * fabs(xc) + nb;
            out = b[c] - ax;
            acc_r += out * out;
            acc_v += v * v;
        }
        r[c] = out;
    }
    __shared__ double sh[2][RB / 32];
    for (int o = 16; o > 0; o >>= 1) {
        acc_r += __shfl_down_sync(0xffffffffu, acc_r, o);
        acc_v += __shfl_down_sync(0xffffffffu, acc_v, o);
    }
    if ((threadIdx.x & 31) == 0) { sh[0][threadIdx.x >> 5] = acc_r; sh[1][threadIdx.x >> 5] = acc_v; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double tr = 0.0, tv = 0.0;
        for (int w = 0; w < RB / 32; w++) { tr += sh[0][w]; tv += sh[1][w]; }
        part[blockIdx.x] = tr;
        part[NRED + blockIdx.x] = tv;
    }
}

// One colour of point red-black SOR on A x = b (the same folded operator as apply_kernel and
// residual_kernel): x_c <- x_c + omega ((b_c - sum_off a_cf x_f) / a_cc - x_c) for the fluid
// interior cells with (i + j + k) % 2 == colour. A folded boundary face contributes +w/3 to a_cc
// and -w/3 to the inward neighbour's coefficient; a plain face -w to a_cc and +w to the
// neighbour's. Within one colour every cell reads only cells of the other colour (the phi ring
// has an even number of meridians), so the parallel pass equals the sequential one.
__global__ void __launch_bounds__(RB)
sor_kernel(const double* __restrict__ b, double* __restrict__ x, const uint8_t* __restrict__ s,
           const GeoIJ* __restrict__ geo, const double* __restrict__ yw, OpC q, int colour,
           double omega) {
    const size_t plane = (size_t)q.jm * q.KP, row = q.KP;
    const size_t NP = (size_t)q.im * plane;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < NP;
         c += (size_t)gridDim.x * blockDim.x) {
        if (!(yw[c] > 0.0)) continue;
        const int k = (int)(c % row);
        const int j = (int)((c / row) % q.jm);
        const int i = (int)(c / plane);
        if (((i + j + k) & 1) != colour) continue;
        const GeoIJ& g = geo[i * q.jm + j];
        const double n1 = q.n1, n2 = g.num2, n3 = g.num3;
        const int kw = (k == 0) ? q.km - 2 : k - 1;
        const int ke = (k == q.km - 2) ? 0 : k + 1;
        double diag = 0.0, off = 0.0;
        if (!s[c + plane]) {
            if (i + 1 == q.im - 1) { diag += n1 * kC13; off -= n1 * kC13 * x[c - plane]; }
            else { diag -= n1; off += n1 * x[c + plane]; }
        }
        if (!s[c - plane]) {
            if (i - 1 == 0) { diag += n1 * kC13; off -= n1 * kC13 * x[c + plane]; }
            else { diag -= n1; off += n1 * x[c - plane]; }
        }
        if (!s[c + row]) {
            if (j + 1 == q.jm - 1) { diag += n2 * kC13; off -= n2 * kC13 * x[c - row]; }
            else { diag -= n2; off += n2 * x[c + row]; }
        }
        if (!s[c - row]) {
            if (j - 1 == 0) { diag += n2 * kC13; off -= n2 * kC13 * x[c + row]; }
            else { diag -= n2; off += n2 * x[c - row]; }
        }
        if (!s[c - k + ke]) { diag -= n3; off += n3 * x[c - k + ke]; }
        if (!s[c - k + kw]) { diag -= n3; off += n3 * x[c - k + kw]; }
        if (diag == 0.0) continue;
        const double xc = x[c];
        x[c] = xc + omega * ((b[c] - off) / diag - xc);
    }
}

// r -= (y.r / y.1) on fluid interior cells: keeps the recursive residual in the range of A
__global__ void reproject_kernel(float* __restrict__ r32, double* __restrict__ r64,
                                 const double* __restrict__ yw, const double* __restrict__ scal,
                                 size_t n) {
    const double mean = scal[11] / scal[6];
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (size_t)gridDim.x * blockDim.x)
        if (yw[c] > 0.0) {
            if (r32) r32[c] -= (float)mean;
            if (r64) r64[c] -= mean;
        }
}

// b (masked copy of the source or the external right-hand side) and p (masked warm start)
__global__ void gather_kernel(const double* __restrict__ src, const double* __restrict__ p_dyn,
                              const double* __restrict__ yw, double* __restrict__ b,
                              double* __restrict__ p, size_t n, int warm) {
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (size_t)gridDim.x * blockDim.x) {
        const bool f = yw[c] > 0.0;
        b[c] = f ? src[c] : 0.0;
        p[c] = (f && warm) ? p_dyn[c] : 0.0;
    }
}

// b -= (y.b / y.1) on fluid interior cells
__global__ void project_kernel(double* __restrict__ b, const double* __restrict__ yw,
                               const double* __restrict__ scal, size_t n) {
    const double mean = scal[5] / scal[6];
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (size_t)gridDim.x * blockDim.x)
        if (yw[c] > 0.0) b[c] -= mean;
}

// p_dyn = p on fluid interior cells, with the y-weighted mean removed when `gauge`
__global__ void scatter_kernel(const double* __restrict__ p, const double* __restrict__ yw,
                               double* __restrict__ p_dyn, const double* __restrict__ scal,
                               size_t n, int gauge) {
    const double mean = gauge ? scal[5] / scal[6] : 0.0;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (size_t)gridDim.x * blockDim.x)
        if (yw[c] > 0.0) p_dyn[c] = p[c] - mean;
}

// ---------------------------------------------------------------------------------------------
template <typename T>
int alloc_vecs(Vecs<T>& v, size_t NP, int jm, int km, int NM, int N, int J, bool krylov) {
    T** big[] = {&v.z, &v.la, &v.lc, &v.lm, &v.b, &v.p, &v.r, &v.d, &v.q};
    const int nbig = krylov ? 9 : 4;        // the FP32 set carries the preconditioner only
    for (int q = 0; q < nbig; q++) {
        ATJUP_CUDA(cudaMalloc(big[q], sizeof(T) * NP));
        ATJUP_CUDA(cudaMemset(*big[q], 0, sizeof(T) * NP));
    }
    ATJUP_CUDA(cudaMalloc(&v.g, sizeof(T) * (size_t)jm * km));
    ATJUP_CUDA(cudaMemset(v.g, 0, sizeof(T) * (size_t)jm * km));
    ATJUP_CUDA(cudaMalloc(&v.gh, sizeof(T) * 2 * (size_t)(NM + 1) * J));
    ATJUP_CUDA(cudaMalloc(&v.cs, sizeof(T) * (size_t)(NM + 1) * N));
    ATJUP_CUDA(cudaMalloc(&v.sn, sizeof(T) * (size_t)(NM + 1) * N));
    ATJUP_CUDA(cudaMalloc(&v.ta, sizeof(T) * (size_t)(NM + 1) * J));
    ATJUP_CUDA(cudaMalloc(&v.tcp, sizeof(T) * (size_t)(NM + 1) * J));
    ATJUP_CUDA(cudaMalloc(&v.tm, sizeof(T) * (size_t)(NM + 1) * J));
    ATJUP_CUDA(cudaMalloc(&v.S3d, sizeof(T) * jm));
    ATJUP_CUDA(cudaMalloc(&v.dj, sizeof(T) * jm));
    return ATJUP_OK;
}

template <typename T>
void free_vecs(Vecs<T>& v) {
    T* all[] = {v.b, v.p, v.r, v.z, v.d, v.q, v.la, v.lc, v.lm, v.g, v.gh, v.cs, v.sn,
                v.ta, v.tcp, v.tm, v.S3d, v.dj};
    for (T* p : all) cudaFree(p);
    v = Vecs<T>();
}

template <typename T>
int upload_setup(Vecs<T>& v, size_t NP, const std::vector<double>& la, const std::vector<double>& lc,
                 const std::vector<double>& lm, const std::vector<double>& cs,
                 const std::vector<double>& sn, const std::vector<double>& ta,
                 const std::vector<double>& tcp, const std::vector<double>& tm,
                 const std::vector<double>& S3d, const std::vector<double>& dj) {
    auto up = [&](T* dst, const std::vector<double>& src) -> int {
        std::vector<T> h(src.begin(), src.end());
        ATJUP_CUDA(cudaMemcpy(dst, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
        return ATJUP_OK;
    };
    int rc;
    if ((rc = up(v.la, la)) || (rc = up(v.lc, lc)) || (rc = up(v.lm, lm)) || (rc = up(v.cs, cs)) ||
        (rc = up(v.sn, sn)) || (rc = up(v.ta, ta)) || (rc = up(v.tcp, tcp)) || (rc = up(v.tm, tm)) ||
        (rc = up(v.S3d, S3d)) || (rc = up(v.dj, dj)))
        return rc;
    (void)NP;
    return ATJUP_OK;
}

// Build y, the line factors and the coarse (column-mode) factors from the mask and geometry.
int setup(AtjupCtx* c, Solver* S) {
    const AtjupParams& P = c->P;
    const int im = P.im, jm = P.jm, km = P.km, KP = c->KP;
    const size_t NP = c->NP;
    S->N = km - 1;
    S->NM = S->N / 2;
    S->J = jm - 2;
    const int N = S->N, NM = S->NM, J = S->J;
    std::vector<uint8_t> s(NP);
    ATJUP_CUDA(cudaMemcpy(s.data(), c->solid, NP, cudaMemcpyDeviceToHost));
    std::vector<GeoIJ> geo((size_t)im * jm);
    ATJUP_CUDA(cudaMemcpy(geo.data(), c->geo, sizeof(GeoIJ) * geo.size(), cudaMemcpyDeviceToHost));
    const double n1 = 1.0 / (P.dr * P.dr);
    auto at = [&](int i, int j, int k) { return ((size_t)i * jm + j) * KP + k; };
    std::vector<double> y(NP, 0.0), la(NP, 0.0), lc(NP, 0.0), lm(NP, 0.0);
    double ysum = 0.0;
    for (int i = 1; i <= im - 2; i++)
        for (int j = 1; j <= jm - 2; j++)
            for (int k = 0; k <= km - 2; k++)
                if (!s[at(i, j, k)]) {
                    const double a = (i == 1 || i == im - 2) ? 1.5 : 1.0;
                    const double d = (j == 1 || j == jm - 2) ? 1.5 : 1.0;
                    y[at(i, j, k)] = a * d;
                    ysum += a * d;
                }
    // radial tridiagonal of A per column: rows = fluid interior cells; diagonal = -(sum of
    // kept faces) plus the fold terms; off-diagonals num1 (fold-modified at i = 1, im-2)
    for (int j = 1; j <= jm - 2; j++)
        for (int k = 0; k <= km - 2; k++) {
            const int kw = (k == 0) ? km - 2 : k - 1, ke = (k == km - 2) ? 0 : k + 1;
            double cprev = 0.0;
            bool prev_fluid = false;
            for (int i = 1; i <= im - 2; i++) {
                const size_t cc = at(i, j, k);
                if (s[cc]) { prev_fluid = false; continue; }
                const GeoIJ& g = geo[(size_t)i * jm + j];
                double den = 0.0, diag = 0.0, lower = 0.0, upper = 0.0;
                if (!s[at(i + 1, j, k)]) {
                    den += n1;
                    if (i + 1 == im - 1) { diag += n1 * kC43; lower += -n1 * kC13; }
                    else upper += n1;
                }
                if (!s[at(i - 1, j, k)]) {
                    den += n1;
                    if (i - 1 == 0) { diag += n1 * kC43; upper += -n1 * kC13; }
                    else lower += n1;
                }
                if (!s[at(i, j + 1, k)]) { den += g.num2; if (j + 1 == jm - 1) diag += g.num2 * kC43; }
                if (!s[at(i, j - 1, k)]) { den += g.num2; if (j - 1 == 0) diag += g.num2 * kC43; }
                if (!s[at(i, j, ke)]) den += g.num3;
                if (!s[at(i, j, kw)]) den += g.num3;
                diag -= den;
                // neighbours outside the run (solid) carry no coupling
                if (!prev_fluid) lower = 0.0;
                if (i + 1 > im - 2 || s[at(i + 1, j, k)]) upper = 0.0;
                const double piv = diag - lower * cprev;
                const double m = 1.0 / piv;
                la[cc] = lower;
                lm[cc] = m;
                lc[cc] = upper * m;
                cprev = lc[cc];
                prev_fluid = true;
            }
        }
    // coarse: S2 = sum_i a_i num2_i, S3_j = sum_i a_i num3_ij (obstacle-free column sums)
    std::vector<double> S3d(jm, 0.0), dj(jm, 0.0);
    double S2 = 0.0;
    for (int i = 1; i <= im - 2; i++) {
        const double a = (i == 1 || i == im - 2) ? 1.5 : 1.0;
        S2 += a * geo[(size_t)i * jm + 1].num2;
    }
    for (int j = 1; j <= jm - 2; j++) {
        double s3 = 0.0;
        for (int i = 1; i <= im - 2; i++) {
            const double a = (i == 1 || i == im - 2) ? 1.5 : 1.0;
            s3 += a * geo[(size_t)i * jm + j].num3;
        }
        S3d[j] = s3;
        dj[j] = (j == 1 || j == jm - 2) ? 1.5 : 1.0;
    }
    std::vector<double> cs((size_t)(NM + 1) * N), sn((size_t)(NM + 1) * N);
    for (int m = 0; m <= NM; m++)
        for (int k = 0; k < N; k++) {
            const double a = 2.0 * M_PI * (double)((long)m * k % N) / N;
            cs[(size_t)m * N + k] = std::cos(a);
            sn[(size_t)m * N + k] = std::sin(a);
        }
    // per wavenumber: rows jj = 0..J-1 (j = jj+1): S2 (e[j+1] + e[j-1] - 2 e[j]) - S3_j lam e[j],
    // folded at both ends (e[0] = 4/3 e[1] - 1/3 e[2]); mode 0: row 0 replaced by e[0] = 0
    std::vector<double> ta((size_t)(NM + 1) * J), tcp((size_t)(NM + 1) * J), tm((size_t)(NM + 1) * J);
    for (int m = 0; m <= NM; m++) {
        const double sl = std::sin(M_PI * m / N);
        const double lam = 4.0 * sl * sl;       // S3_j already carries 1 / dphi^2
        double cprev = 0.0;
        for (int jj = 0; jj < J; jj++) {
            const int j = jj + 1;
            double a = S2, b = -2.0 * S2 - S3d[j] * lam, cu = S2;
            if (jj == 0) { b += kC43 * S2; cu -= kC13 * S2; a = 0.0; }
            if (jj == J - 1) { b += kC43 * S2; a -= kC13 * S2; cu = 0.0; }
            if (m == 0 && jj == 0) { a = 0.0; b = 1.0; cu = 0.0; }
            const double piv = b - a * cprev;
            const double mm = 1.0 / piv;
            ta[(size_t)m * J + jj] = a;
            tm[(size_t)m * J + jj] = mm;
            tcp[(size_t)m * J + jj] = cu * mm;
            cprev = tcp[(size_t)m * J + jj];
        }
    }
    int rc;
    if ((rc = alloc_vecs(S->v64, NP, jm, km, NM, N, J, true))) return rc;
    if ((rc = alloc_vecs(S->v32, NP, jm, km, NM, N, J, false))) return rc;
    if ((rc = upload_setup(S->v64, NP, la, lc, lm, cs, sn, ta, tcp, tm, S3d, dj))) return rc;
    if ((rc = upload_setup(S->v32, NP, la, lc, lm, cs, sn, ta, tcp, tm, S3d, dj))) return rc;
    ATJUP_CUDA(cudaMalloc(&S->yw, sizeof(double) * NP));
    ATJUP_CUDA(cudaMemcpy(S->yw, y.data(), sizeof(double) * NP, cudaMemcpyHostToDevice));
    ATJUP_CUDA(cudaMalloc(&S->part, sizeof(double) * NRED * 2 + sizeof(double) * 64 * 1024));
    ATJUP_CUDA(cudaMalloc(&S->scal, sizeof(double) * 16));
    ATJUP_CUDA(cudaMemset(S->scal, 0, sizeof(double) * 16));
    ATJUP_CUDA(cudaMallocHost(&S->hs, sizeof(double) * 16));
    c->yw_sum = ysum;
    S->ready = true;
    return ATJUP_OK;
}

Solver* get_solver(AtjupCtx* c) { return reinterpret_cast<Solver*>(c->solver); }

// One preconditioned CG solve of A x = rhs, x from zero, to ||r|| <= tol ||rhs||. The Krylov
// vectors (V.b = rhs, V.p = x, r, d, q) are FP64; the preconditioner (radial lines and column
// modes, set M) runs in precision T. Returns iterations; *rel = final recursive ||r|| / ||rhs||.
template <typename T>
int pcg(AtjupCtx* c, Solver* S, Vecs<double>& V, Vecs<T>& M, double tol, int max_iter, int* iters,
        double* rel) {
    const AtjupParams& P = c->P;
    const size_t NP = c->NP;
    OpC q{P.im, P.jm, P.km, c->KP, 1.0 / (P.dr * P.dr)};
    cudaStream_t st = c->stream;
    const int nb = NRED;
    double* part = S->part;
    double* part2 = S->part + 2 * NRED;      // partials of the inverse DFT (J * blocks)
    const int kblocks = (S->N + 127) / 128;
    // r = b (x = 0), ||b||
    ATJUP_CUDA(cudaMemcpyAsync(V.r, V.b, sizeof(double) * NP, cudaMemcpyDeviceToDevice, st));
    ATJUP_CUDA(cudaMemsetAsync(V.p, 0, sizeof(double) * NP, st));
    dot_kernel<double, double><<<nb, RB, 0, st>>>(V.r, V.r, nullptr, NP, part); c->launches++;
    finalize_kernel<<<1, 1, 0, st>>>(part, nb, S->scal, 7, 0); c->launches++;
    ATJUP_CUDA(cudaMemcpyAsync(S->hs, S->scal, sizeof(double) * 16, cudaMemcpyDeviceToHost, st));
    ATJUP_CUDA(cudaStreamSynchronize(st));
    const double bnorm = std::sqrt(S->hs[7]);
    *iters = 0;
    *rel = 0.0;
    if (bnorm == 0.0) return ATJUP_OK;
    auto precond = [&](int first) -> int {
        line_kernel<T><<<dim3((P.km - 1 + 127) / 128, P.jm - 2), 128, 0, st>>>(
            V.r, M.z, M.la, M.lc, M.lm, S->yw, M.g, q);
        dft_fwd_kernel<T><<<dim3((S->NM + 1 + 127) / 128, S->J), 128, 0, st>>>(
            M.g, M.cs, M.sn, M.gh, S->N, S->NM, S->J, P.km);
        theta_solve_kernel<T><<<dim3((S->NM + 1 + 63) / 64, 2), 64, 0, st>>>(
            M.gh, M.ta, M.tcp, M.tm, M.dj, S->NM, S->J, S->N);
        dft_inv_kernel<T><<<dim3(kblocks, S->J), 128, 0, st>>>(M.gh, M.cs, M.sn, M.z, V.r, S->yw,
                                                               M.lm, q, S->N, S->NM, S->J, part2);
        finalize_kernel<<<1, 1, 0, st>>>(part2, kblocks * S->J, S->scal, 8, first ? 0 : 2);
        c->launches += 5;
        if (first) {   // rho = y r z
            ATJUP_CUDA(cudaMemcpyAsync(S->scal + 0, S->scal + 8, sizeof(double), cudaMemcpyDeviceToDevice, st));
        }
        return ATJUP_OK;
    };
    int rc;
    if ((rc = precond(1))) return rc;
    direction_kernel<T><<<nb, RB, 0, st>>>(V.d, M.z, S->scal, NP, 1); c->launches++;
    const int check = 4;
    double rr = bnorm * bnorm;
    int it = 0;
    for (it = 1; it <= max_iter; it++) {
        apply_kernel<double><<<nb, RB, 0, st>>>(V.d, V.q, c->solid, c->geo, S->yw, q, part);
        finalize_kernel<<<1, 1, 0, st>>>(part, nb, S->scal, 4, 1);
        update_kernel<double><<<nb, RB, 0, st>>>(V.p, V.r, V.d, V.q, S->scal, NP, part);
        finalize_kernel<<<1, 1, 0, st>>>(part, nb, S->scal, 3, 0);
        c->launches += 4;
        if ((rc = precond(0))) return rc;
        direction_kernel<T><<<nb, RB, 0, st>>>(V.d, M.z, S->scal, NP, 0); c->launches++;
        if (it % check == 0 || it == max_iter) {
            // drop the rounding drift of r out of the range of A (its y-component)
            dot_kernel<double, double><<<nb, RB, 0, st>>>(S->yw, V.r, nullptr, NP, part);
            finalize_kernel<<<1, 1, 0, st>>>(part, nb, S->scal, 11, 0);
            reproject_kernel<<<nb, RB, 0, st>>>(nullptr, V.r, S->yw, S->scal, NP);
            c->launches += 3;
            ATJUP_CUDA(cudaMemcpyAsync(S->hs, S->scal, sizeof(double) * 16, cudaMemcpyDeviceToHost, st));
            ATJUP_CUDA(cudaStreamSynchronize(st));
            rr = S->hs[3];
            if (!std::isfinite(rr)) { set_error("pressure_solve: non-finite residual"); return ATJUP_ERR_NONFINITE; }
            if (std::sqrt(rr) <= tol * bnorm) break;
        }
    }
    ATJUP_CUDA(cudaGetLastError());
    *iters = std::min(it, max_iter);
    *rel = std::sqrt(rr) / bnorm;
    return ATJUP_OK;
}

}  // namespace

void solver_free(AtjupCtx* c) {
    Solver* S = get_solver(c);
    if (!S) return;
    free_vecs(S->v64);
    free_vecs(S->v32);
    cudaFree(S->part);
    cudaFree(S->scal);
    cudaFree(S->yw);
    if (S->hs) cudaFreeHost(S->hs);
    delete S;
    c->solver = nullptr;
}

int pressure_residual_solve(AtjupCtx* c, const AtjupSolveOpts* o, AtjupSolveStats* st) {
    const AtjupParams& P = c->P;
    if (!(o->rel_tol > 0.0) || o->max_iter < 1) { set_error("pressure_solve: bad tolerance or cap"); return ATJUP_ERR_ARG; }
    if (o->external_rhs && !c->solve_b) { set_error("pressure_solve: no external right-hand side set"); return ATJUP_ERR_ARG; }
    Solver* S = get_solver(c);
    int rc;
    if (!S) {
        S = new Solver();
        c->solver = S;
        if ((rc = setup(c, S))) { solver_free(c); return rc; }
    }
    cudaStream_t stm = c->stream;
    const size_t NP = c->NP;
    const int nb = NRED;
    OpC q{P.im, P.jm, P.km, c->KP, 1.0 / (P.dr * P.dr)};
    // right-hand side: the reference's clamped divergence source, or the caller's b
    const double* src = c->src;
    if (o->external_rhs) src = c->solve_b;
    else {
        if ((rc = launch_prepare_projection(c))) return rc;
        if ((rc = launch_pressure_source(c))) return rc;
    }
    Vecs<double>& V = S->v64;
    double* b64 = c->tmp;    // the projected right-hand side (FP64), kept for the refinement
    double* p64 = c->tmp2;   // the FP64 solution
    const int warm = o->external_rhs ? 0 : 1;
    gather_kernel<<<nb, RB, 0, stm>>>(src, c->f[ATJUP_F_P_DYN], S->yw, b64, p64, NP, warm);
    // compatibility: remove the y-component of b
    dot_kernel<double, double><<<nb, RB, 0, stm>>>(S->yw, b64, nullptr, NP, S->part);
    finalize_kernel<<<1, 1, 0, stm>>>(S->part, nb, S->scal, 5, 0);
    {
        std::vector<double> one(1, c->yw_sum);
        ATJUP_CUDA(cudaMemcpyAsync(S->scal + 6, one.data(), sizeof(double), cudaMemcpyHostToDevice, stm));
        ATJUP_CUDA(cudaStreamSynchronize(stm));
    }
    project_kernel<<<nb, RB, 0, stm>>>(b64, S->yw, S->scal, NP);
    dot_kernel<double, double><<<nb, RB, 0, stm>>>(b64, b64, nullptr, NP, S->part);
    finalize_kernel<<<1, 1, 0, stm>>>(S->part, nb, S->scal, 9, 0);
    c->launches += 6;
    ATJUP_CUDA(cudaMemcpyAsync(S->hs, S->scal, sizeof(double) * 16, cudaMemcpyDeviceToHost, stm));
    ATJUP_CUDA(cudaStreamSynchronize(stm));
    const double bnorm = std::sqrt(S->hs[9]);
    int total_it = 0, inner = 0;
    double rel = 0.0, floor_rel = 0.0, prev = 1e300;
    const bool mixed = (o->precision == ATJUP_PREC_MIXED);
    // Iterative refinement with the residual formed in FP64: r = b - A p; solve A e = r by PCG
    // with FP64 Krylov vectors (the preconditioner in FP32 for the mixed form: the operator's
    // condition number, ~1e9, is above 1/eps of FP32, so FP32 can carry the preconditioner -- whose
    // radial-line and column-mode systems have condition numbers ~1e5 -- but not the residual);
    // p += e. Stops at the tolerance, or when the residual no longer falls (it has reached the
    // rounding floor of an FP64 p, which is reported).
    if (o->mode == ATJUP_SOLVE_SOR) {
        // point red-black SOR with omega, the residual checked every `check` sweeps
        const double omega = (o->omega > 0.0 && o->omega < 2.0) ? o->omega : 1.0;
        const int check = 50;
        int sweeps = 0;
        for (;;) {
            residual_kernel<<<nb, RB, 0, stm>>>(b64, p64, V.b, c->solid, c->geo, S->yw, q, S->part);
            finalize_kernel<<<1, 1, 0, stm>>>(S->part, nb, S->scal, 10, 0);
            finalize_kernel<<<1, 1, 0, stm>>>(S->part + NRED, nb, S->scal, 12, 0);
            c->launches += 3;
            ATJUP_CUDA(cudaMemcpyAsync(S->hs, S->scal, sizeof(double) * 16, cudaMemcpyDeviceToHost, stm));
            ATJUP_CUDA(cudaStreamSynchronize(stm));
            rel = (bnorm > 0.0) ? std::sqrt(S->hs[10]) / bnorm : 0.0;
            floor_rel = (bnorm > 0.0) ? 2.220446049250313e-16 * std::sqrt(S->hs[12]) / bnorm : 0.0;
            if (!std::isfinite(rel)) { set_error("pressure_solve: non-finite residual"); return ATJUP_ERR_NONFINITE; }
            if (rel <= o->rel_tol || sweeps >= o->max_iter) break;
            const int n = std::min(check, o->max_iter - sweeps);
            for (int t = 0; t < n; t++) {
                sor_kernel<<<nb, RB, 0, stm>>>(b64, p64, c->solid, c->geo, S->yw, q, 0, omega);
                sor_kernel<<<nb, RB, 0, stm>>>(b64, p64, c->solid, c->geo, S->yw, q, 1, omega);
            }
            c->launches += 2 * n;
            sweeps += n;
        }
        total_it = sweeps;
    }
    const int max_outer = (o->mode == ATJUP_SOLVE_SOR) ? -1 : 8;
    for (int outer = 0; outer <= max_outer; outer++) {
        residual_kernel<<<nb, RB, 0, stm>>>(b64, p64, V.b, c->solid, c->geo, S->yw, q, S->part);
        finalize_kernel<<<1, 1, 0, stm>>>(S->part, nb, S->scal, 10, 0);
        finalize_kernel<<<1, 1, 0, stm>>>(S->part + NRED, nb, S->scal, 12, 0);
        c->launches += 3;
        ATJUP_CUDA(cudaMemcpyAsync(S->hs, S->scal, sizeof(double) * 16, cudaMemcpyDeviceToHost, stm));
        ATJUP_CUDA(cudaStreamSynchronize(stm));
        rel = (bnorm > 0.0) ? std::sqrt(S->hs[10]) / bnorm : 0.0;
        floor_rel = (bnorm > 0.0) ? 2.220446049250313e-16 * std::sqrt(S->hs[12]) / bnorm : 0.0;
        if (!std::isfinite(rel)) { set_error("pressure_solve: non-finite residual"); return ATJUP_ERR_NONFINITE; }
        if (rel <= o->rel_tol || total_it >= o->max_iter || outer == max_outer) break;
        if (outer > 0 && rel > 0.5 * prev) break;            // stalled at the FP64 floor
        prev = rel;
        int it = 0;
        double inner_rel = 0.0;
        const int budget = o->max_iter - total_it;
        const double tgt = o->rel_tol * bnorm / std::max(std::sqrt(S->hs[10]), 1e-300);
        const double itol = std::min(1e-3, std::max(0.5 * tgt, 1e-12));
        if (mixed) rc = pcg<float>(c, S, V, S->v32, itol, budget, &it, &inner_rel);
        else rc = pcg<double>(c, S, V, V, itol, budget, &it, &inner_rel);
        if (rc) return rc;
        add_kernel<<<nb, RB, 0, stm>>>(p64, V.p, NP);
        c->launches++;
        total_it += it;
        inner++;
    }
    // write the solution into p_dyn (fluid interior cells), fix the gauge for a cold start, fold
    if (o->external_rhs) {
        dot_kernel<double, double><<<nb, RB, 0, stm>>>(S->yw, p64, nullptr, NP, S->part);
        finalize_kernel<<<1, 1, 0, stm>>>(S->part, nb, S->scal, 5, 0);
        c->launches += 2;
    }
    scatter_kernel<<<nb, RB, 0, stm>>>(p64, S->yw, c->f[ATJUP_F_P_DYN], S->scal, NP, o->external_rhs ? 1 : 0);
    c->launches++;
    if ((rc = launch_pressure_fold(c, c->f[ATJUP_F_P_DYN]))) return rc;
    ATJUP_CUDA(cudaGetLastError());
    if (st) {
        st->iterations = total_it;
        st->inner_solves = inner;
        st->rel_residual = rel;
        st->b_norm = bnorm;
        st->rel_floor = floor_rel;
    }
    // converged: at the tolerance, or within a small factor of the FP64 floor above it
    if (rel > o->rel_tol && rel > 8.0 * floor_rel) {
        char msg[160];
        snprintf(msg, sizeof(msg), "pressure_solve: relative residual %.3e above tolerance %.1e "
                 "(FP64 floor %.2e) after %d iterations", rel, o->rel_tol, floor_rel, total_it);
        set_error(msg);
        return ATJUP_ERR_NOT_CONVERGED;
    }
    return ATJUP_OK;
}

}  // namespace atjup
