// The in-loop projection of the horizontal wind around the obstacle (projectAroundObstacle with
// in_loop = true, InitValues_Jup.cpp:1595-1822; called every ATJUP_CONE_PROJ_STRIDE iterations
// after the column balance of v, cJupiterModel.cpp:1356-1363).
//
// Per level i in 1..im-2 that holds solid cells, a box M cells wider than the obstacle's
// cross-section (clipped to j 1..jm-2, k 1..km-2, phi = 0 on a one-cell halo) and up to two SOR
// solves on it: with ATJUP_CONE_PROJ_DIV = H > 0 first the divergence solve (the cells within H
// cells, Chebyshev in 3-D, of the body take the 3-D face divergence s r D of the flow before the
// correction as a source and close their wall faces), then the wall-flux solve (a wall face
// carries the prescribed flux -U.n). Each solve is warm-started from its own phi of the previous
// call, runs lexicographic SOR (omega 1.9) until the largest change of a sweep is at most 1e-10
// of the largest |phi| (at most 40000 sweeps), and increments v and w by the average of the two
// face corrections of each direction (a wall face's correction is minus the cell's velocity).
// Finally the seam column k = km-1 takes v and w of k = 0.
//
// B200 form. One thread block per level; the level's phi, the cell flags and the per-cell
// constants sit in shared memory (about 170 KB for the 105 x 117 box of the 41 x 181 x 361 grid).
// Lexicographic SOR is replayed exactly as a pipelined wavefront: cell (a, b) of the box lies on
// the anti-diagonal d = a + b, its sweep-t update needs sweep t of (a-1, b) and (a, b-1) and sweep
// t-1 of (a+1, b) and (a, b+1), so step tau of the wavefront updates diagonal d = tau - 2(t-1)
// for every sweep t in flight at once -- about D/2 diagonals of D = NJ + NK - 2 per step instead
// of one. Each sweep meets one diagonal per step, so the warp that owns that diagonal reduces the
// sweep's largest change and largest |phi| without atomics, and sweep t is complete after step
// D + 2(t-1), where its stopping test is taken. The sweeps after the converged one have by then
// already updated the first diagonals; the block restores the newest snapshot of phi that
// precedes them (one every SNAP_EVERY steps, in HBM) and replays up to the converged sweep. The
// arithmetic is the reference's, operation for operation (this file is compiled without FMA
// contraction), so the result is the reference's to the bit.
#include <algorithm>
#include <cmath>
#include <vector>

#include "ctx.cuh"

namespace atjup {

namespace {

constexpr double CONE_OMEGA = 1.9;       // InitValues_Jup.cpp:1726
constexpr int CONE_MAXIT = 40000;        // InitValues_Jup.cpp:1728
constexpr double CONE_TOL = 1.0e-10;     // InitValues_Jup.cpp:1761
constexpr int SNAP_EVERY = 64;           // wavefront steps between snapshots
constexpr int CONE_THREADS = 1024;
constexpr size_t CONE_SMEM_CAP = 200 * 1024;

// cell flags of the box (uint32 per cell: these bits, the special-cell index above bit 6)
enum : uint32_t { CF_SOLID = 1, CF_N = 2, CF_S = 4, CF_W = 8, CF_E = 16, CF_NEAR = 32 };

}  // namespace

struct ConeLevel {
    int i, jlo, klo, NJ, NK, PJ, D, n_spec;
    int64_t info_off;   // uint32 [NJ * PJ]: flags | special index << 6
    int64_t spec_off;   // int32 [n_spec]: box cell a * PJ + b of each special cell
    int64_t phi_off;    // double [(NJ + 2) * PJ] per warm-start buffer (halo included)
    int64_t snap_off;   // double [n_snap * (NJ + 2) * PJ]
    int64_t tab_off;    // double [2 * n_spec] (global-memory mode)
    int64_t row_off;    // double [5 * NJ]: aN, aS, aL, s, s dphi (global-memory mode)
    int n_snap, ring;
};

struct ConeState {
    std::vector<ConeLevel> lv;
    ConeLevel* d_lv = nullptr;
    uint32_t* info = nullptr;
    int32_t* spec = nullptr;
    double* prev[2] = {nullptr, nullptr};   // 0: divergence solve, 1: wall-flux solve
    double* snap = nullptr;
    double* tab = nullptr;
    double* rows = nullptr;
    double* s = nullptr;                    // [jm] max(sinthe_min, |sin(the_j)|)
    int* stats = nullptr;                   // [2 * levels] sweeps of the last call
    int H = 0, M = 0;
    size_t smem = 0;                        // dynamic shared memory per block (0: global mode)
    bool allocated = false;
    int64_t n_info = 0, n_spec = 0, n_phi = 0, n_snap = 0, n_tab = 0, n_row = 0;
};

namespace {

struct ConeArgs {
    const ConeLevel* lv;
    const uint32_t* info;
    const int32_t* spec;
    double* prev0;
    double* prev1;
    double* snap;
    double* tab;
    double* rows;
    const double* s;
    int* stats;
    const double* u;
    double* v;
    double* w;
    const uint8_t* solid;
    const double* rad;
    int jm, km, KP, H, smem_mode;
    double dr, dthe, dphi;
};

// One SOR update of box cell (a, b) (InitValues_Jup.cpp:1739-1758), in the reference's order of
// operations; returns false for a cell the sweep skips (solid, or no fluid face: A = 0).
__device__ __forceinline__ bool cone_update(double* phi, const uint32_t* info, const double* tab,
                                            const double* rows, int NJ, int PJ, int a, int b,
                                            bool div, double dthe, double dphi, double& dch,
                                            double& pabs) {
    const uint32_t inf = info[a * PJ + b];
    if (inf & CF_SOLID) return false;
    const int q = (a + 1) * PJ + (b + 1);
    const double aN = rows[a], aS = rows[NJ + a], aL = rows[2 * NJ + a];
    double A = 0.0, B = 0.0;
    if (div && (inf & CF_NEAR)) {
        if (!(inf & CF_N)) { A += aN; B += aN * phi[q - PJ]; }
        if (!(inf & CF_S)) { A += aS; B += aS * phi[q + PJ]; }
        if (!(inf & CF_W)) { A += aL; B += aL * phi[q - 1]; }
        if (!(inf & CF_E)) { A += aL; B += aL * phi[q + 1]; }
        B += tab[2 * (inf >> 6)];
    } else {
        double vp = 0.0, wp = 0.0;
        if (inf & (CF_N | CF_S | CF_W | CF_E)) { vp = tab[2 * (inf >> 6)]; wp = tab[2 * (inf >> 6) + 1]; }
        const double sj = rows[3 * NJ + a];
        if (inf & CF_N) B -= aN * dthe * (-vp); else { A += aN; B += aN * phi[q - PJ]; }
        if (inf & CF_S) B -= aS * dthe * (vp);  else { A += aS; B += aS * phi[q + PJ]; }
        if (inf & CF_W) B -= aL * sj * dphi * (-wp); else { A += aL; B += aL * phi[q - 1]; }
        if (inf & CF_E) B -= aL * sj * dphi * (wp);  else { A += aL; B += aL * phi[q + 1]; }
    }
    if (!(A > 0.0)) return false;
    const double p = phi[q];
    const double pn = p + CONE_OMEGA * (B / A - p);
    dch = fmax(dch, fabs(pn - p));
    phi[q] = pn;
    pabs = fmax(pabs, fabs(pn));
    return true;
}

__device__ __forceinline__ double warp_max(double x) {
    for (int o = 16; o; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
    return x;
}

// One wavefront step tau: every sweep t in [t_lo, t_hi] updates its diagonal tau - 2(t-1). With
// ring != nullptr each sweep's largest change and |phi| are folded into ring[t % R].
__device__ void cone_step(double* phi, const uint32_t* info, const double* tab, const double* rows,
                          int NJ, int NK, int PJ, int D, int tau, int t_stop, bool div,
                          double dthe, double dphi, double* ring, int R) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    const int t_hi = min(t_stop, tau / 2 + 1);
    const int t_lo = tau <= D ? 1 : (tau - D + 1) / 2 + 1;
    for (int t = t_lo + warp; t <= t_hi; t += nwarps) {
        const int d = tau - 2 * (t - 1);
        const int a0 = max(0, d - (NK - 1)), a1 = min(d, NJ - 1);
        double dch = 0.0, pabs = 0.0;
        for (int a = a0 + lane; a <= a1; a += 32)
            cone_update(phi, info, tab, rows, NJ, PJ, a, d - a, div, dthe, dphi, dch, pabs);
        if (ring) {
            dch = warp_max(dch);
            pabs = warp_max(pabs);
            if (lane == 0) {
                double* r = ring + 2 * (t % R);
                if (d == 0) { r[0] = dch; r[1] = pabs; }
                else { r[0] = fmax(r[0], dch); r[1] = fmax(r[1], pabs); }
            }
        }
    }
}

// s r D of a cell within H cells of the body: its 3-D face divergence with face values the
// average of the two cells and zero through a face to a solid cell (InitValues_Jup.cpp:1653-1664).
__device__ double cone_face_div(const ConeArgs& A, int i, int j, int k) {
    const size_t row = (size_t)A.jm * A.KP;
    const size_t c = ((size_t)i * A.jm + j) * A.KP + k;
    const double r = A.rad[i], rp = r + 0.5 * A.dr, rm = r - 0.5 * A.dr;
    const double sj = A.s[j], sp = 0.5 * (sj + A.s[j + 1]), sm = 0.5 * (sj + A.s[j - 1]);
    const double up = A.solid[c + row] ? 0.0 : 0.5 * (A.u[c] + A.u[c + row]);
    const double um = A.solid[c - row] ? 0.0 : 0.5 * (A.u[c] + A.u[c - row]);
    const double vp = A.solid[c + A.KP] ? 0.0 : 0.5 * (A.v[c] + A.v[c + A.KP]);
    const double vm = A.solid[c - A.KP] ? 0.0 : 0.5 * (A.v[c] + A.v[c - A.KP]);
    const double wp = A.solid[c + 1] ? 0.0 : 0.5 * (A.w[c] + A.w[c + 1]);
    const double wm = A.solid[c - 1] ? 0.0 : 0.5 * (A.w[c] + A.w[c - 1]);
    return sj * r * (rp * rp * up - rm * rm * um) / (r * r * A.dr) + (sp * vp - sm * vm) / A.dthe +
           (wp - wm) / A.dphi;
}

__device__ void cone_copy(double* dst, const double* src, int n) {
    for (int x = threadIdx.x; x < n; x += blockDim.x) dst[x] = src[x];
}

// Lexicographic SOR of one level's solve as the pipelined wavefront; returns the reference's
// sweep count `it` (the converged sweep, or CONE_MAXIT + 1 without convergence).
__device__ int cone_sor(double* phi, const uint32_t* info, const double* tab, const double* rows,
                        int NJ, int NK, int PJ, int D, bool div, double dthe, double dphi,
                        double* ring, int R, double* snap, int n_snap, int* snap_tag) {
    const int nphi = (NJ + 2) * PJ;
    cone_copy(snap, phi, nphi);
    if (threadIdx.x == 0) {
        snap_tag[0] = -1;
        for (int s = 1; s < n_snap; s++) snap_tag[s] = INT_MIN;
    }
    __syncthreads();
    int next = 1 % n_snap, t_conv = 0, it = CONE_MAXIT + 1;
    for (int tau = 0;; tau++) {
        cone_step(phi, info, tab, rows, NJ, NK, PJ, D, tau, CONE_MAXIT, div, dthe, dphi, ring, R);
        __syncthreads();
        if (tau >= D && ((tau - D) & 1) == 0) {
            const int t = (tau - D) / 2 + 1;       // the sweep this step completed
            const double* r = ring + 2 * (t % R);
            if (r[0] <= CONE_TOL * fmax(r[1], 1.0e-30)) { t_conv = t; break; }
            if (t == CONE_MAXIT) break;
        }
        if (tau % SNAP_EVERY == SNAP_EVERY - 1) {
            cone_copy(snap + (size_t)next * nphi, phi, nphi);
            if (threadIdx.x == 0) snap_tag[next] = tau;
            next = (next + 1) % n_snap;
            __syncthreads();
        }
    }
    if (t_conv > 0) {
        // back to the newest snapshot in which no cell is past sweep t_conv, then replay with
        // the sweeps capped at t_conv up to the step that completes it
        it = t_conv;
        const int target = 2 * (t_conv - 1), tau_c = D + 2 * (t_conv - 1);
        int best = 0, btag = INT_MIN;
        for (int s = 0; s < n_snap; s++)
            if (snap_tag[s] != INT_MIN && snap_tag[s] <= target && snap_tag[s] > btag) { best = s; btag = snap_tag[s]; }
        cone_copy(phi, snap + (size_t)best * nphi, nphi);
        __syncthreads();
        for (int tau = btag + 1; tau <= tau_c; tau++) {
            cone_step(phi, info, tab, rows, NJ, NK, PJ, D, tau, t_conv, div, dthe, dphi, nullptr, R);
            __syncthreads();
        }
    }
    return it;
}

__global__ void __launch_bounds__(CONE_THREADS, 1) cone_kernel(ConeArgs A) {
    extern __shared__ __align__(16) unsigned char cone_smem[];
    __shared__ int snap_tag[64];
    const ConeLevel L = A.lv[blockIdx.x];
    const int NJ = L.NJ, NK = L.NK, PJ = L.PJ, D = L.D, i = L.i;
    const int nphi = (NJ + 2) * PJ;
    double *phi, *tab, *rows, *ring;
    const uint32_t* info;
    if (A.smem_mode) {
        phi = reinterpret_cast<double*>(cone_smem);
        tab = phi + nphi;
        rows = tab + 2 * L.n_spec;
        ring = rows + 5 * NJ;
        uint32_t* inf = reinterpret_cast<uint32_t*>(ring + 2 * L.ring);
        for (int x = threadIdx.x; x < NJ * PJ; x += blockDim.x) inf[x] = A.info[L.info_off + x];
        info = inf;
    } else {
        phi = nullptr;
        tab = A.tab + L.tab_off;
        rows = A.rows + L.row_off;
        ring = reinterpret_cast<double*>(cone_smem);
        info = A.info + L.info_off;
    }
    // the row coefficients (InitValues_Jup.cpp:1733-1735)
    for (int a = threadIdx.x; a < NJ; a += blockDim.x) {
        const int j = L.jlo + a;
        const double sj = A.s[j];
        rows[a] = 0.5 * (sj + A.s[j - 1]) / (A.dthe * A.dthe);
        rows[NJ + a] = 0.5 * (sj + A.s[j + 1]) / (A.dthe * A.dthe);
        rows[2 * NJ + a] = 1.0 / (sj * A.dphi * A.dphi);
        rows[3 * NJ + a] = sj;
        rows[4 * NJ + a] = sj * A.dphi;
    }
    const int32_t* spec = A.spec + L.spec_off;
    if (A.H == 0 && threadIdx.x == 0) A.stats[2 * blockIdx.x] = 0;
    for (int pass = A.H > 0 ? 0 : 1; pass < 2; pass++) {
        const bool div = pass == 0;
        double* prev = (div ? A.prev0 : A.prev1) + L.phi_off;
        if (A.smem_mode) cone_copy(phi, prev, nphi);
        else phi = prev;
        // the per-cell constants: the source of the divergence solve from the flow before it,
        // the wall-face velocities of the wall-flux solve from the flow it starts from
        __syncthreads();
        for (int x = threadIdx.x; x < L.n_spec; x += blockDim.x) {
            const int cb = spec[x], a = cb / PJ, b = cb - a * PJ;
            const int j = L.jlo + a, k = L.klo + b;
            if (div) {
                tab[2 * x] = (info[cb] & CF_NEAR) ? cone_face_div(A, i, j, k) : 0.0;
            } else {
                const size_t c = ((size_t)i * A.jm + j) * A.KP + k;
                tab[2 * x] = A.v[c];
                tab[2 * x + 1] = A.w[c];
            }
        }
        __syncthreads();
        const int it = cone_sor(phi, info, tab, rows, NJ, NK, PJ, D, div, A.dthe, A.dphi, ring,
                                L.ring, A.snap + L.snap_off, L.n_snap, snap_tag);
        // v and w incremented by the average of the two face corrections (InitValues_Jup.cpp:
        // 1785-1793), a wall face's correction being minus the cell's velocity
        for (int x = threadIdx.x; x < NJ * NK; x += blockDim.x) {
            const int a = x / NK, b = x - a * NK;
            const uint32_t inf = info[a * PJ + b];
            if (inf & CF_SOLID) continue;
            const size_t c = ((size_t)i * A.jm + (L.jlo + a)) * A.KP + (L.klo + b);
            const int q = (a + 1) * PJ + (b + 1);
            const double vp = A.v[c], wp = A.w[c], pp = phi[q];
            const double sd = rows[4 * NJ + a];
            const double dN = (inf & CF_N) ? -vp : (pp - phi[q - PJ]) / A.dthe;
            const double dS = (inf & CF_S) ? -vp : (phi[q + PJ] - pp) / A.dthe;
            const double dW = (inf & CF_W) ? -wp : (pp - phi[q - 1]) / sd;
            const double dE = (inf & CF_E) ? -wp : (phi[q + 1] - pp) / sd;
            A.v[c] = vp + 0.5 * (dN + dS);
            A.w[c] = wp + 0.5 * (dW + dE);
        }
        // the warm start of the next call
        if (A.smem_mode) cone_copy(prev, phi, nphi);
        if (threadIdx.x == 0) A.stats[2 * blockIdx.x + pass] = it;
        __syncthreads();
    }
}

// the seam copy: v and w of k = km-1 from k = 0 in every (i, j) row (InitValues_Jup.cpp:1806-1807)
__global__ void cone_seam_kernel(double* v, double* w, int rows, int km, int KP) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    v[(size_t)r * KP + km - 1] = v[(size_t)r * KP];
    w[(size_t)r * KP + km - 1] = w[(size_t)r * KP];
}

}  // namespace

void cone_free(AtjupCtx* c) {
    ConeState* cs = static_cast<ConeState*>(c->cone);
    if (!cs) return;
    cudaFree(cs->d_lv);
    cudaFree(cs->info);
    cudaFree(cs->spec);
    cudaFree(cs->prev[0]);
    cudaFree(cs->prev[1]);
    cudaFree(cs->snap);
    cudaFree(cs->tab);
    cudaFree(cs->rows);
    cudaFree(cs->s);
    cudaFree(cs->stats);
    delete cs;
    c->cone = nullptr;
}

// The static part, once per grid: the levels that cut the obstacle with their boxes, the cell
// flags (solid, solid neighbours along j and k, within H cells of the body), the list of cells
// that carry a constant (wall or near cells), and the buffers: the warm starts of both solves
// (zero until the first call, as the reference's per-level phi_prev), the snapshots, the stats.
// The solid mask and sin(the_j) are read back from the device copies set_grid made.
int cone_prepare(AtjupCtx* c) {
    if (c->cone) return ATJUP_OK;
    if (!c->grid_set) { set_error("cone projection: set_grid first"); return ATJUP_ERR_ARG; }
    const AtjupParams& P = c->P;
    if (P.cone_proj_margin < 0 || P.cone_proj_div < 0) {
        set_error("cone projection: margin and div must be >= 0");
        return ATJUP_ERR_ARG;
    }
    const int im = P.im, jm = P.jm, km = P.km, KP = c->KP;
    std::vector<uint8_t> sol(c->NP);
    std::vector<double> sinthe(jm);
    ATJUP_CUDA(cudaMemcpyAsync(sol.data(), c->solid, c->NP, cudaMemcpyDeviceToHost, c->stream));
    ATJUP_CUDA(cudaMemcpyAsync(sinthe.data(), c->sin_the, sizeof(double) * jm, cudaMemcpyDeviceToHost, c->stream));
    ATJUP_CUDA(cudaStreamSynchronize(c->stream));
    auto S = [&](int i, int j, int k) { return sol[((size_t)i * jm + j) * KP + k] != 0; };
    std::vector<double> s(jm);
    for (int j = 0; j < jm; j++) s[j] = std::max(P.sinthe_min, std::fabs(sinthe[j]));
    const int H = P.cone_proj_div, M = P.cone_proj_margin;
    // within H cells (Chebyshev, 3-D, clipped to the grid) of a solid cell: a separable dilation
    // of the solid mask along k, j and i (InitValues_Jup.cpp:1634-1646)
    const size_t N = (size_t)im * jm * km;
    std::vector<uint8_t> near;
    if (H > 0) {
        std::vector<uint8_t> a(N), b(N);
        for (int i = 0; i < im; i++)
            for (int j = 0; j < jm; j++)
                for (int k = 0; k < km; k++) a[((size_t)i * jm + j) * km + k] = S(i, j, k);
        auto dilate = [&](const std::vector<uint8_t>& in, std::vector<uint8_t>& out, int axis) {
            const int n[3] = {im, jm, km};
            const size_t stride[3] = {(size_t)jm * km, (size_t)km, 1};
            for (int i = 0; i < im; i++)
                for (int j = 0; j < jm; j++)
                    for (int k = 0; k < km; k++) {
                        const int x[3] = {i, j, k};
                        const size_t at = ((size_t)i * jm + j) * km + k;
                        uint8_t v = 0;
                        for (int d = -H; d <= H && !v; d++) {
                            const int y = x[axis] + d;
                            if (y >= 0 && y < n[axis]) v = in[at + (ptrdiff_t)d * (ptrdiff_t)stride[axis]];
                        }
                        out[at] = v;
                    }
        };
        dilate(a, b, 2);
        dilate(b, a, 1);
        dilate(a, b, 0);
        near.swap(b);
    }
    auto* cs = new ConeState();
    cs->H = H;
    cs->M = M;
    std::vector<uint32_t> info;
    std::vector<int32_t> spec;
    int64_t n_phi = 0, n_snap = 0, n_tab = 0, n_row = 0;
    size_t smem_max = 0, ring_bytes = 0;
    for (int i = 1; i < im - 1; i++) {
        int jmin = jm, jmax = -1, kmin = km, kmax = -1;
        for (int j = 0; j < jm; j++)
            for (int k = 0; k < km; k++)
                if (S(i, j, k)) {
                    jmin = std::min(jmin, j); jmax = std::max(jmax, j);
                    kmin = std::min(kmin, k); kmax = std::max(kmax, k);
                }
        if (jmax < 0) continue;                      // above the body
        const int jlo = std::max(1, jmin - M), jhi = std::min(jm - 2, jmax + M);
        const int klo = std::max(1, kmin - M), khi = std::min(km - 2, kmax + M);
        if (jhi < jlo || khi < klo) continue;        // no cell in the box
        ConeLevel L{};
        L.i = i; L.jlo = jlo; L.klo = klo;
        L.NJ = jhi - jlo + 1; L.NK = khi - klo + 1;
        L.PJ = (L.NK + 2 + 1) & ~1;                  // even: the diagonal stride PJ-1 is odd
        L.D = L.NJ + L.NK - 2;
        L.ring = L.D / 2 + 2;
        L.n_snap = (L.D + SNAP_EVERY) / SNAP_EVERY + 2;
        if (L.n_snap > 64) { delete cs; set_error("cone projection: box too large"); return ATJUP_ERR_UNSUPPORTED; }
        L.info_off = (int64_t)info.size();
        L.spec_off = (int64_t)spec.size();
        info.resize(info.size() + (size_t)L.NJ * L.PJ, CF_SOLID);
        for (int a = 0; a < L.NJ; a++)
            for (int b = 0; b < L.NK; b++) {
                const int j = jlo + a, k = klo + b;
                uint32_t f = 0;
                if (S(i, j, k)) f = CF_SOLID;
                else {
                    if (S(i, j - 1, k)) f |= CF_N;
                    if (S(i, j + 1, k)) f |= CF_S;
                    if (S(i, j, k - 1)) f |= CF_W;
                    if (S(i, j, k + 1)) f |= CF_E;
                    if (H > 0 && near[((size_t)i * jm + j) * km + k]) f |= CF_NEAR;
                    if (f) {
                        f |= (uint32_t)(spec.size() - L.spec_off) << 6;
                        spec.push_back(a * L.PJ + b);
                    }
                }
                info[L.info_off + (size_t)a * L.PJ + b] = f;
            }
        L.n_spec = (int)(spec.size() - L.spec_off);
        const int64_t nphi = (int64_t)(L.NJ + 2) * L.PJ;
        L.phi_off = n_phi;  n_phi += nphi;
        L.snap_off = n_snap; n_snap += (int64_t)L.n_snap * nphi;
        L.tab_off = n_tab;  n_tab += 2 * (int64_t)L.n_spec;
        L.row_off = n_row;  n_row += 5 * (int64_t)L.NJ;
        const size_t sm = sizeof(double) * ((size_t)nphi + 2 * (size_t)L.n_spec + 5 * (size_t)L.NJ +
                                            2 * (size_t)L.ring) + sizeof(uint32_t) * (size_t)L.NJ * L.PJ;
        smem_max = std::max(smem_max, sm);
        ring_bytes = std::max(ring_bytes, sizeof(double) * 2 * (size_t)L.ring);
        cs->lv.push_back(L);
    }
    c->cone = cs;
    const bool smem_mode = smem_max <= CONE_SMEM_CAP;
    cs->smem = smem_mode ? smem_max : ring_bytes;
    cs->n_phi = n_phi;
    const size_t nl = cs->lv.size();
    ATJUP_CUDA(cudaMalloc(&cs->s, sizeof(double) * jm));
    ATJUP_CUDA(cudaMemcpy(cs->s, s.data(), sizeof(double) * jm, cudaMemcpyHostToDevice));
    ATJUP_CUDA(cudaMalloc(&cs->stats, sizeof(int) * 2 * std::max<size_t>(nl, 1)));
    ATJUP_CUDA(cudaMemset(cs->stats, 0, sizeof(int) * 2 * std::max<size_t>(nl, 1)));
    if (nl == 0) return ATJUP_OK;
    ATJUP_CUDA(cudaMalloc(&cs->d_lv, sizeof(ConeLevel) * nl));
    ATJUP_CUDA(cudaMemcpy(cs->d_lv, cs->lv.data(), sizeof(ConeLevel) * nl, cudaMemcpyHostToDevice));
    ATJUP_CUDA(cudaMalloc(&cs->info, sizeof(uint32_t) * info.size()));
    ATJUP_CUDA(cudaMemcpy(cs->info, info.data(), sizeof(uint32_t) * info.size(), cudaMemcpyHostToDevice));
    ATJUP_CUDA(cudaMalloc(&cs->spec, sizeof(int32_t) * std::max<size_t>(spec.size(), 1)));
    if (!spec.empty())
        ATJUP_CUDA(cudaMemcpy(cs->spec, spec.data(), sizeof(int32_t) * spec.size(), cudaMemcpyHostToDevice));
    for (double*& p : cs->prev) {
        ATJUP_CUDA(cudaMalloc(&p, sizeof(double) * n_phi));
        ATJUP_CUDA(cudaMemset(p, 0, sizeof(double) * n_phi));
    }
    ATJUP_CUDA(cudaMalloc(&cs->snap, sizeof(double) * n_snap));
    if (!smem_mode) {
        ATJUP_CUDA(cudaMalloc(&cs->tab, sizeof(double) * std::max<int64_t>(n_tab, 1)));
        ATJUP_CUDA(cudaMalloc(&cs->rows, sizeof(double) * n_row));
    }
    ATJUP_CUDA(cudaFuncSetAttribute(cone_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cs->smem));
    return ATJUP_OK;
}

// One in-loop projection on the context's stream (v and w in place).
int launch_cone_projection(AtjupCtx* c) {
    if (int rc = cone_prepare(c)) return rc;
    const AtjupParams& P = c->P;
    ConeState* cs = static_cast<ConeState*>(c->cone);
    if (!cs->lv.empty()) {
        ConeArgs A{};
        A.lv = cs->d_lv; A.info = cs->info; A.spec = cs->spec;
        A.prev0 = cs->prev[0]; A.prev1 = cs->prev[1]; A.snap = cs->snap;
        A.tab = cs->tab; A.rows = cs->rows; A.s = cs->s; A.stats = cs->stats;
        A.u = c->f[ATJUP_F_U]; A.v = c->f[ATJUP_F_V]; A.w = c->f[ATJUP_F_W];
        A.solid = c->solid; A.rad = c->rad;
        A.jm = P.jm; A.km = P.km; A.KP = c->KP; A.H = cs->H;
        A.smem_mode = cs->tab == nullptr;
        A.dr = P.dr; A.dthe = P.dthe; A.dphi = P.dphi;
        c->launches++;
        cone_kernel<<<(unsigned)cs->lv.size(), CONE_THREADS, cs->smem, c->stream>>>(A);
        ATJUP_CHECK_LAUNCH("cone projection");
    }
    const int rows = P.im * P.jm;
    c->launches++;
    cone_seam_kernel<<<(rows + 255) / 256, 256, 0, c->stream>>>(c->f[ATJUP_F_V], c->f[ATJUP_F_W], rows, P.km, c->KP);
    ATJUP_CHECK_LAUNCH("cone seam");
    return ATJUP_OK;
}

}  // namespace atjup

using namespace atjup;

extern "C" {

int atjup_gpu_cone_project(AtjupCtx* c) {
    if (!c) return ATJUP_ERR_ARG;
    if (!c->grid_set) { set_error("cone_project: set_grid first"); return ATJUP_ERR_ARG; }
    return launch_cone_projection(c);
}

int atjup_gpu_cone_stats(AtjupCtx* c, int32_t* level_i, int32_t* sweeps, int32_t cap, int32_t* n_levels) {
    if (!c || !n_levels) return ATJUP_ERR_ARG;
    if (int rc = cone_prepare(c)) return rc;
    ConeState* cs = static_cast<ConeState*>(c->cone);
    const int nl = (int)cs->lv.size();
    *n_levels = nl;
    const int n = std::min(nl, std::max(cap, 0));
    if (n == 0) return ATJUP_OK;
    std::vector<int> st(2 * (size_t)nl);
    ATJUP_CUDA(cudaMemcpyAsync(st.data(), cs->stats, sizeof(int) * st.size(), cudaMemcpyDeviceToHost, c->stream));
    ATJUP_CUDA(cudaStreamSynchronize(c->stream));
    for (int l = 0; l < n; l++) {
        if (level_i) level_i[l] = cs->lv[l].i;
        if (sweeps) { sweeps[2 * l] = st[2 * l]; sweeps[2 * l + 1] = st[2 * l + 1]; }
    }
    return ATJUP_OK;
}

}  // extern "C"
