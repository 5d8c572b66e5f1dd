// RK4 time step of the dynamics: buoyancy level mean, hydrostatic column integral, the fused
// RHS + stage kernel, and the mixture density.
//
// Reference: cJupiterModel::RungeKuttaJup (RungeKutta_Jup_Turb.cpp:261-583) with RHSJup
// (RHS_Jup_Turb.cpp:31-1457). The reference runs every stage as two passes over the grid (RHS
// everywhere into rhs_*, then accumulate and form the next stage input) and copies y -> y_n after
// the step. Here one kernel per stage reads the stage input X_s (7-point stencil), the time-level
// n state Y and the accumulator at the cell, and writes X_{s+1} and the accumulator; stage 3
// writes Y itself. Non-integrated cells (radial walls, the three rows next to each pole, the
// seam copy k = km-1, solid cells) keep their start-of-step values: stages 0-2 copy Y into
// X_{s+1} there, which is what the reference's untouched live fields hold. The stage kernel
// marches a tile of columns up through the radial planes; each plane's inputs reach shared memory
// two planes ahead as tensor-memory-accelerator copies (cp.async.bulk.tensor on mbarriers).
#include "ctx.cuh"

#include <cuda.h>

#include <cstring>

namespace atjup {
namespace {

// Block tile: TK meridians x TJ colatitude rows, marching through a chunk of the radial planes.
// The tiles cover the km-1 = 360 distinct meridians exactly (10 x 36); the seam copy k = km-1 is
// never read by a stage (the ring wraps 359 -> 0) and is left alone.
constexpr int TK = 36, TJ = 7, NT = 256, NL = TK * TJ;   // 252 live threads of 256
constexpr int NCH = 2;   // radial chunks per column tile (the step: 6.69 ms, 6.72 with 3 or 4)
constexpr int HJ = TJ + 2;                               // halo rows of a tile
constexpr int NX = 5;    // FP64 per-cell inputs besides Y: rho, wall_nue, nue, Q_rad, Q_precip

// Per-cell flags, precomputed from the static mask (atjup_gpu_set_grid): bit 0 solid, 1 solid i+1,
// 2 solid i-1, 3 solid j+1, 4 solid j-1, 5 solid k+1 (ring), 6 solid k-1 (ring), 7 integrated
// (i in [1, im-2], j in [3, jm-4], k in [0, km-2], not solid).
enum : uint8_t { NB_S = 1, NB_IP = 2, NB_IM = 4, NB_JP = 8, NB_JM = 16, NB_KP = 32, NB_KM = 64,
                 NB_INT = 128 };

struct StageConst {
    int im, jm, km, KP;
    int stage;
    double c_in, wgt, dt, one_sixth;
    double inv_2dr, inv_2dthe, inv_2dphi, inv_dr2, inv_dthe2, inv_dphi2;
    double cor_phi_f;          // (nd_cor * 2) * omega
    double coeff_energy_p;     // u_0^2 / (cp_mix t_ref)
    double to_nd, r_mix, rR, g, t_ref, R_mix, cp_mix, u_0, L_rad;
    double t_visc;             // t_diff_scale / (re pr)
    double inv_re;
    double buoy_k;             // -nd_buoy * buoy_scale * buoy_ramp * buoyancy
    double metric_on, cor_rad_on, Coriolis, centrifugal, pgrad_scale;
    double rad_coupling, precip_coupling, turb_coupling;
    int pgrad_wall, adiabatic, adiabatic_rho, hydro_split, use_hp, cell_hold;
    int has_nue, has_heating, precip_local;
    // FP64 step: the accumulator is written once, at stage 2, from the right-hand sides of stages
    // 0 and 1 recovered as (X_{s+1} - y_n) / c_s (X1 read per cell, X2 the stage's own input; the
    // subtraction is exact, X lying within a factor 2 of y_n) plus stage 2's own: stages 0 and 1
    // neither write nor read it
    int acc_free;
    double inv_c_half;         // 1 / c_in of stages 0 and 1 (2 / dt)
};

// The stage buffers X (stage input), Xo (next stage input) and acc are typed by the kernel's
// template arguments (FP64, or FP32 in the mixed step); Y (time level n), the pressures and the
// frozen inputs are FP64.
struct StagePtrs {
    const void* X[4];
    const void* X1[4];         // stage 2 with acc_free: the stage-1 input (X1), read per cell
    void* Xo[4];
    double* Y[4];
    void* acc[4];
    const double *p_dyn, *p_hydro, *p_stat, *rho, *wall_nue, *nue, *Q_rad, *Q_precip;
    double *aux_u, *aux_v, *aux_w;
    const uint8_t* nb;
    const GeoIJ* geo;
    const double* buoy_ref;
    const double *cell_vbar0, *cell_ubar0;
};

// The halo tiles of the stage input (t, u, v, w) and of p_dyn, p_hydro are copied by the tensor
// memory accelerator: one cp.async.bulk.tensor per field and plane, issued by one thread, its
// completion counted on the ring slot's mbarrier. A box starts on a 16-byte boundary, OX columns
// before the tile (k0 - OX; OX = 2 doubles or 4 floats), and is TK + 2 OX wide and HJ rows high
// (j0 - 1 .. j0 + TJ; rows outside the grid arrive as zeros, and only cells that are never
// integrated read them). Boxes are padded to 128 bytes in shared memory.
template <typename T>
struct Box3 {
    static constexpr int OX = 16 / (int)sizeof(T);
    static constexpr int W = TK + 2 * OX;
    static constexpr int BYTES = W * HJ * (int)sizeof(T);
    static constexpr int PAD = (BYTES + 127) / 128 * 128 / (int)sizeof(T);
};

// The per-cell inputs (no halo) are boxes of TK x TJ x 1 at (k0, j0, i): their shared-memory
// layout [TJ][TK] is the block's thread order, and k0 (a multiple of 36) is a 16-byte boundary.
template <typename T>
struct CellBox {
    static constexpr int BYTES = TK * TJ * (int)sizeof(T);
};

// The tensor maps of one launch, all over [im][jm][KP] arrays: the stage input's four fields and
// p_dyn, p_hydro (halo boxes), and the per-cell inputs (cell boxes; only those the stage reads are
// encoded)
struct __align__(64) StageMaps {
    CUtensorMap x[4];
    CUtensorMap p[2];
    CUtensorMap ps;            // p_stat
    CUtensorMap y[4];          // time-level-n t, u, v, w (stages 1-3)
    CUtensorMap ax[4];         // the accumulator, or X1 at stage 2 of the FP64 step
    CUtensorMap ex[NX];        // rho, wall_nue, nue, Q_rad, Q_precip
};

template <typename TI, typename TA>
struct __align__(128) StageSmem {
    TI tile[3][4][Box3<TI>::PAD];            // stage input t, u, v, w of planes i, i+1, i+2
    double ptile[3][2][Box3<double>::PAD];   // p_dyn, p_hydro of the same planes
    double ps[3][NT];         // p_stat at the cells of the same three planes
    double Yx[2][4][NT];      // time-level-n t, u, v, w of planes i and i+1 (stages 1-3)
    double ex[2][NX][NT];     // FP64 per-cell inputs of planes i and i+1
    TA ax[2][4][NT];          // accumulators of planes i and i+1 (stages 1-3)
    GeoIJ geo[2][TJ];         // geometry rows of planes i and i+1
    double cm[2][2][TJ];      // cell-hold means (v, u) of planes i and i+1
    uint8_t nb[2][NT];        // per-cell flags of planes i and i+1
    unsigned long long bar[4];    // the barrier of each halo ring slot (three used)
    unsigned long long barx[2];   // the barrier of each per-cell slot
};
// two blocks per SM: 228 KB of shared memory per SM, 1 KB of it reserved per block
static_assert(2 * (sizeof(StageSmem<double, double>) + 1024) <= 233472, "two FP64 stage blocks per SM");

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

__device__ __forceinline__ double ld(const double* p) { return __ldg(p); }

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

// one tensor copy of the box at (x, y, z) of map into dst, counted on the barrier bar
__device__ __forceinline__ void tma3(void* dst, const CUtensorMap* map, unsigned bar, int x, int y,
                                     int z) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3, %4}], [%5];\n"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z),
          "r"(bar) : "memory");
}
__device__ __forceinline__ void expect_bytes(unsigned bar, unsigned bytes) {
    // the fence orders the block's earlier plain writes to the slot (the seam patches) before the
    // copies' writes
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes)
                 : "memory");
}

// One thread: the tensor copies of plane i's six halo boxes and its p_stat into ring slot i % 3,
// their bytes expected on the slot's barrier.
template <typename TI, typename TA>
__device__ __forceinline__ void issue_boxes(StageSmem<TI, TA>& S, const StageMaps& M, int i,
                                            int j0, int k0) {
    const int sl = i % 3;
    const unsigned bar = smem_u32(&S.bar[sl]);
    expect_bytes(bar, 4 * Box3<TI>::BYTES + 2 * Box3<double>::BYTES + CellBox<double>::BYTES);
#pragma unroll
    for (int f = 0; f < 4; f++) tma3(S.tile[sl][f], &M.x[f], bar, k0 - Box3<TI>::OX, j0 - 1, i);
#pragma unroll
    for (int f = 0; f < 2; f++) tma3(S.ptile[sl][f], &M.p[f], bar, k0 - Box3<double>::OX, j0 - 1, i);
    tma3(S.ps[sl], &M.ps, bar, k0, j0, i);
}

// One thread: the tensor copies of plane i's per-cell inputs into slot i % 2 (the time-level-n
// state and the accumulator or X1 where the stage reads them, rho, wall_nue, and nue and the
// heating rates when present).
template <typename TI, typename TA>
__device__ __forceinline__ void issue_cells(StageSmem<TI, TA>& S, const StageMaps& M,
                                            const StageConst& q, int i, int j0, int k0) {
    const int sl = i & 1;
    const unsigned bar = smem_u32(&S.barx[sl]);
    const bool need_y = q.stage > 0, need_ax = q.stage > 0 && (!q.acc_free || q.stage >= 2);
    unsigned bytes = 2 * CellBox<double>::BYTES;
    if (need_y) bytes += 4 * CellBox<double>::BYTES;
    if (need_ax) bytes += 4 * CellBox<TA>::BYTES;
    if (q.has_nue) bytes += CellBox<double>::BYTES;
    if (q.has_heating) bytes += 2 * CellBox<double>::BYTES;
    expect_bytes(bar, bytes);
    if (need_y)
        for (int f = 0; f < 4; f++) tma3(S.Yx[sl][f], &M.y[f], bar, k0, j0, i);
    if (need_ax)
        for (int f = 0; f < 4; f++) tma3(S.ax[sl][f], &M.ax[f], bar, k0, j0, i);
    tma3(S.ex[sl][0], &M.ex[0], bar, k0, j0, i);
    tma3(S.ex[sl][1], &M.ex[1], bar, k0, j0, i);
    if (q.has_nue) tma3(S.ex[sl][2], &M.ex[2], bar, k0, j0, i);
    if (q.has_heating) {
        tma3(S.ex[sl][3], &M.ex[3], bar, k0, j0, i);
        tma3(S.ex[sl][4], &M.ex[4], bar, k0, j0, i);
    }
}

// Wait for slot sl's copies (phase parity par), at most TMA_SPIN polls; false when they did not
// arrive (the block then abandons the stage and poisons its cells).
constexpr int TMA_SPIN = 1 << 22;
__device__ __forceinline__ bool wait_boxes(const unsigned long long* bar, unsigned par) {
    const unsigned a = smem_u32(bar);
    for (int n = 0; n < TMA_SPIN; n++) {
        unsigned ok;
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                     " selp.u32 %0, 1, 0, p;\n}\n" : "=r"(ok) : "r"(a), "r"(par) : "memory");
        if (ok) return true;
    }
    return false;
}

// The ring of km-1 meridians: the box's column of k = -1 (left tile) takes k = km-2, and the
// column of k = km-1 (the tile holding km-2) takes k = 0. Patch thread t < 54 of the left tile, or
// 64 <= t < 118 of the right, owns field (t mod 64) / 9, row (t mod 64) % 9 of that column:
// wrap_src reads its value from global memory, wrap_put stores it into the landed box.
__device__ __forceinline__ int wrap_role(int tid, int k0, const StageConst& q) {
    const int t = tid & 63;
    if (t >= 54) return -1;
    if (tid < 64) return k0 == 0 ? t : -1;
    if (tid < 128) return (k0 + TK >= q.km - 1) ? 64 + t : -1;
    return -1;
}
template <typename TI>
__device__ __forceinline__ double wrap_src(const StagePtrs& a, const StageConst& q, int role, int i,
                                           int j0) {
    const int t = role & 63, f = t / 9, r = t % 9;
    int j = j0 - 1 + r;
    j = j < 0 ? 0 : (j > q.jm - 1 ? q.jm - 1 : j);
    const size_t o = ((size_t)i * q.jm + j) * q.KP + (role < 64 ? q.km - 2 : 0);
    if (f < 4) return (double)static_cast<const TI*>(a.X[f])[o];
    return (f == 4 ? a.p_dyn : a.p_hydro)[o];
}
template <typename TI, typename TA>
__device__ __forceinline__ void wrap_put(StageSmem<TI, TA>& S, const StageConst& q, int role,
                                         int i, int k0, double v) {
    const int t = role & 63, f = t / 9, r = t % 9, sl = i % 3;
    if (f < 4) {
        const int col = role < 64 ? Box3<TI>::OX - 1 : Box3<TI>::OX + (q.km - 1 - k0);
        S.tile[sl][f][r * Box3<TI>::W + col] = (TI)v;
    } else {
        const int col = role < 64 ? Box3<double>::OX - 1 : Box3<double>::OX + (q.km - 1 - k0);
        S.ptile[sl][f - 4][r * Box3<double>::W + col] = v;
    }
}

// Issue the copies of plane i's flags, geometry rows and cell means into slot i % 2 (small, or
// bytes whose rows do not start on 16-byte boundaries: plain asynchronous copies).
template <typename TI, typename TA>
__device__ __forceinline__ void issue_extra(StageSmem<TI, TA>& S, const StagePtrs& a,
                                            const StageConst& q, int i, int j0, int k0, int tid) {
    const int sl = i & 1;
    // flags: 4 bytes per copy along a tile row (k0 and the row pitch are multiples of 4)
    if (tid < TJ * (TK / 4) && k0 + 4 * (tid % (TK / 4)) <= q.km - 2) {
        const int ty = tid / (TK / 4), kq = tid % (TK / 4);
        const int j = min(j0 + ty, q.jm - 1);
        cp_async4(&S.nb[sl][ty * TK + 4 * kq], a.nb + ((size_t)i * q.jm + j) * q.KP + k0 + 4 * kq);
    }
    // geometry rows (sizeof(GeoIJ) / 8 doubles per row) and the cell-hold means
    constexpr int GD = (int)(sizeof(GeoIJ) / 8);
    for (int e = tid; e < TJ * GD; e += NT) {
        const int r = e / GD, f = e % GD;
        const int j = min(j0 + r, q.jm - 1);
        cp_async8(reinterpret_cast<double*>(&S.geo[sl][r]) + f,
                  reinterpret_cast<const double*>(a.geo + (size_t)i * q.jm + j) + f);
    }
    if (q.cell_hold && tid < 2 * TJ) {
        const int f = tid / TJ, r = tid % TJ;
        const int j = min(j0 + r, q.jm - 1);
        cp_async8(&S.cm[sl][f][r], (f == 0 ? a.cell_vbar0 : a.cell_ubar0) + (size_t)i * q.jm + j);
    }
}

// One RK stage: every (j, k) column of the block's tile, plane by plane. TI is the storage of the
// stage input, TO of the next stage input, TA of the accumulators, R the arithmetic of the
// right-hand side (all double in the FP64 step; the mixed step stores the buffers in FP32 --
// stage 0 <double, float, float> reads the FP64 state, stages 1-3 <float, float, float> -- and
// evaluates the stencils in FP32). Kept in FP64 in both: the differences of the FP64 pressures
// p_dyn, p_hydro and p_stat (then rounded to R), the buoyancy anomaly against the FP64 level
// mean, the heating rates of the FP64 sources, the next stage input y_n + c_in rhs and the final
// update y_n + dt/6 acc from the FP64 time-level-n state, and the projection source aux.
template <typename TI, typename TO, typename TA, typename R>
__global__ void __launch_bounds__(NT, 2)
rk_stage_kernel(StagePtrs a, StageConst q, const __grid_constant__ StageMaps M) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    StageSmem<TI, TA>& S = *reinterpret_cast<StageSmem<TI, TA>*>(smem_raw);
    const int tid = threadIdx.x;
    const int tx = tid % TK, ty = tid / TK;
    const int k0 = blockIdx.x * TK, j0 = blockIdx.y * TJ;
    const int k = k0 + tx, j = j0 + ty;
    const bool live = (tid < NL) && (k <= q.km - 2) && (j < q.jm);
    const size_t row = (size_t)q.KP, plane = (size_t)q.jm * row;
    constexpr int WT = Box3<TI>::W, WP = Box3<double>::W;   // row pitch of the boxes
    const int hT = (ty + 1) * WT + (tx + Box3<TI>::OX);      // this cell in a stage-input box
    const int hP = (ty + 1) * WP + (tx + Box3<double>::OX);  // this cell in a pressure box
    // radial chunk [i_lo, i_hi); the march starts one plane below to fill the radial window
    const int per = (q.im + NCH - 1) / NCH;
    const int i_lo = blockIdx.z * per, i_hi = min(q.im, i_lo + per);
    const int i_st = (i_lo > 0) ? i_lo - 1 : 0;
    const int role = wrap_role(tid, k0, q);

    if (tid == 0) {
        for (int sl = 0; sl < 3; sl++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&S.bar[sl])) : "memory");
        for (int sl = 0; sl < 2; sl++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&S.barx[sl])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    // per ring slot: copies in flight, and the parity of their phase (halo ring, per-cell ring)
    unsigned pend = 0, par = 0, pendx = 0, parx = 0;
    if (tid == 0) {
        issue_boxes(S, M, i_st, j0, k0);
        if (i_st + 1 < q.im) issue_boxes(S, M, i_st + 1, j0, k0);
        issue_cells(S, M, q, i_st, j0, k0);
    }
    pend |= 1u << (i_st % 3);
    if (i_st + 1 < q.im) pend |= 1u << ((i_st + 1) % 3);
    pendx |= 1u << (i_st & 1);
    issue_extra(S, a, q, i_st, j0, k0, tid);
    cp_commit();
    cp_commit();
    double wnext = 0.0;           // a seam thread's value for the next plane to land

    // radial window: the cell's values in plane i-1 (t, u, v, w, p_dyn, p_stat)
    double m_t = 0.0, m_u = 0.0, m_v = 0.0, m_w = 0.0, m_pd = 0.0, m_ps = 0.0;

    for (int i = i_st; i < i_hi; i++) {
        const bool next2 = i + 2 < q.im && i + 2 <= i_hi;
        if (next2) {
            if (tid == 0) issue_boxes(S, M, i + 2, j0, k0);
            pend |= 1u << ((i + 2) % 3);
        }
        if (i + 1 < i_hi) {
            if (tid == 0) issue_cells(S, M, q, i + 1, j0, k0);
            pendx |= 1u << ((i + 1) & 1);
            issue_extra(S, a, q, i + 1, j0, k0, tid);
        }
        cp_commit();
        cp_wait1();
        // the boxes of planes i and i+1 not waited for yet, then their seam columns (planes
        // i_st and i_st + 1 read directly, later ones prefetched a plane ahead)
        bool lost = false;
        for (int p = i; p <= i + 1; p++) {
            const int sl = p % 3;
            if (!(pend >> sl & 1u)) continue;
            if (!wait_boxes(&S.bar[sl], par >> sl & 1u)) lost = true;
            pend &= ~(1u << sl);
            par ^= 1u << sl;
            if (role >= 0 && !lost) {
                wrap_put(S, q, role, p, k0, p <= i_st + 1 ? wrap_src<TI>(a, q, role, p, j0) : wnext);
                asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
            }
        }
        if (role >= 0 && next2) wnext = wrap_src<TI>(a, q, role, i + 2, j0);
        // plane i's per-cell boxes
        if (pendx >> (i & 1) & 1u) {
            if (!wait_boxes(&S.barx[i & 1], parx >> (i & 1) & 1u)) lost = true;
            pendx &= ~(1u << (i & 1));
            parx ^= 1u << (i & 1);
        }
        if (__syncthreads_or(lost)) {
            // the copies still in flight (each wait bounded), then every cell of the chunk NaN
            for (int sl = 0; sl < 3; sl++)
                if (pend >> sl & 1u) wait_boxes(&S.bar[sl], par >> sl & 1u);
            for (int sl = 0; sl < 2; sl++)
                if (pendx >> sl & 1u) wait_boxes(&S.barx[sl], parx >> sl & 1u);
            asm volatile("cp.async.wait_all;\n" ::: "memory");
            if (live)
                for (int ip = i_lo; ip < i_hi; ip++) {
                    const size_t c = (size_t)ip * plane + (size_t)j * row + k;
                    for (int f = 0; f < 4; f++) {
                        if (q.stage < 3) static_cast<TO*>(a.Xo[f])[c] = (TO)__longlong_as_double(0x7ff8000000000000LL);
                        else a.Y[f][c] = __longlong_as_double(0x7ff8000000000000LL);
                    }
                }
            return;
        }

        const int cs = i % 3, ns = (i + 1) % 3, xs = i & 1;
        const TI* Tt = S.tile[cs][0];
        const TI* Ut = S.tile[cs][1];
        const TI* Vt = S.tile[cs][2];
        const TI* Wt = S.tile[cs][3];
        const double* Pt = S.ptile[cs][0];
        const double* Ht = S.ptile[cs][1];
        if (live && i >= i_lo) {
            const size_t c = (size_t)i * plane + (size_t)j * row + k;
            const uint8_t nbm = S.nb[xs][tid];
            if (!(nbm & NB_INT)) {
                if (q.stage == 0) {
#pragma unroll
                    for (int f = 0; f < 4; f++) static_cast<TO*>(a.Xo[f])[c] = (TO)ld(a.Y[f] + c);
                } else if (q.stage < 3) {
#pragma unroll
                    for (int f = 0; f < 4; f++) static_cast<TO*>(a.Xo[f])[c] = (TO)S.Yx[xs][f][tid];
                }
            } else {
                const GeoIJ& g = S.geo[xs][ty];
                const R t0 = (R)Tt[hT], u0 = (R)Ut[hT], v0 = (R)Vt[hT];
                const R w0 = (R)Wt[hT];
                const TI* Tn = S.tile[ns][0];
                const TI* Un = S.tile[ns][1];
                const TI* Vn = S.tile[ns][2];
                const TI* Wn = S.tile[ns][3];
                // first and second centred differences (RHS_Jup_Turb.cpp:180-254); exp_rm = 1
#define DERIVS(F, FN, FM, f0, d1r, d2r, d1t, d2t, d1p, d2p)                           \
    const R d1r = ((R)FN[hT] - (R)FM) * (R)q.inv_2dr;                                 \
    const R d2r = ((R)FN[hT] - (R)2.0 * f0 + (R)FM) * (R)q.inv_dr2;                   \
    const R d1t = ((R)F[hT + WT] - (R)F[hT - WT]) * (R)q.inv_2dthe;                   \
    const R d2t = ((R)F[hT + WT] - (R)2.0 * f0 + (R)F[hT - WT]) * (R)q.inv_dthe2;     \
    const R d1p = ((R)F[hT + 1] - (R)F[hT - 1]) * (R)q.inv_2dphi;                     \
    const R d2p = ((R)F[hT + 1] - (R)2.0 * f0 + (R)F[hT - 1]) * (R)q.inv_dphi2;
                DERIVS(Tt, Tn, m_t, t0, dtdr, d2tdr2, dtdthe, d2tdthe2, dtdphi, d2tdphi2)
                DERIVS(Ut, Un, m_u, u0, dudr, d2udr2, dudthe, d2udthe2, dudphi, d2udphi2)
                DERIVS(Vt, Vn, m_v, v0, dvdr, d2vdr2, dvdthe, d2vdthe2, dvdphi, d2vdphi2)
                DERIVS(Wt, Wn, m_w, w0, dwdr, d2wdr2, dwdthe, d2wdthe2, dwdphi, d2wdphi2)
#undef DERIVS
                // pressure gradients, solid faces mirrored to the local value (RHS_Jup_Turb.cpp:119-130)
                const bool wall = q.pgrad_wall;
                const double pc = Pt[hP];
                const double pip = (wall && (nbm & NB_IP)) ? pc : S.ptile[ns][0][hP];
                const double pim = (wall && (nbm & NB_IM)) ? pc : m_pd;
                const double pjp = (wall && (nbm & NB_JP)) ? pc : Pt[hP + WP];
                const double pjm = (wall && (nbm & NB_JM)) ? pc : Pt[hP - WP];
                const double pkp = (wall && (nbm & NB_KP)) ? pc : Pt[hP + 1];
                const double pkm = (wall && (nbm & NB_KM)) ? pc : Pt[hP - 1];
                const R dpdr = (R)((pip - pim) * q.inv_2dr);
                const R dpdthe = (R)((pjp - pjm) * q.inv_2dthe);
                const R dpdphi = (R)((pkp - pkm) * q.inv_2dphi);

                // body forces (RHS_Jup_Turb.cpp:384-423)
                const R Coriolis_rad = (R)g.cor_rad * w0;
                const R Coriolis_the = (R)g.cor_the * w0;
                R v_cor = v0, u_cor = u0;
                if (q.cell_hold) {
                    v_cor -= (R)S.cm[xs][0][ty];
                    u_cor -= (R)S.cm[xs][1][ty];
                }
                const R Coriolis_phi = (R)q.cor_phi_f * (+(R)g.costhe * v_cor + (R)g.sinthe_true * u_cor);
                const R v_invrm = v0 * (R)g.inv_rm;
                const R w_invrs = w0 * (R)g.inv_rmsinthe;

                // compression work with the hydrostatic part (RHS_Jup_Turb.cpp:459-482)
                const double rho_l = S.ex[xs][0][tid];
                double dpstatdr64 = 0.0;
                if (q.adiabatic) {
                    dpstatdr64 = (S.ps[ns][tid] - m_ps) * q.inv_2dr * q.to_nd;
                    if (q.adiabatic_rho && rho_l > 0.0 && isfinite(rho_l)) dpstatdr64 *= q.r_mix / rho_l;
                }
                const R dpstatdr = (R)dpstatdr64;
                const R pressure_t = (R)q.coeff_energy_p *
                    (u0 * (dpdr + dpstatdr) + v_invrm * dpdthe + w_invrs * dpdphi);
                const R transport_t = u0 * dtdr + v_invrm * dtdthe + w_invrs * dtdphi;
                const R transport_u = u0 * dudr + v_invrm * dudthe + w_invrs * dudphi -
                                      (R)q.metric_on * (v0 * v0 + w0 * w0) * (R)g.inv_rm;
                const R transport_v = u0 * dvdr + v_invrm * dvdthe + w_invrs * dvdphi +
                                      (u0 * v0 - w0 * w0 * (R)g.cotanthe) * (R)g.inv_rm;
                const R transport_w = u0 * dwdr + v_invrm * dwdthe + w_invrs * dwdphi +
                                      (w0 * u0 + v0 * w0 * (R)g.cotanthe) * (R)g.inv_rm;

                // diffusion (RHS_Jup_Turb.cpp:521-545)
#define G_(x) ((R)g.x)
                const R two_inv_rm = (R)2.0 * G_(inv_rm);
                const R diffusion_t = d2tdr2 + dtdr * two_inv_rm + d2tdthe2 * G_(inv_rm2) +
                                      dtdthe * G_(costhe_inv_rm2sinthe) + d2tdphi2 * G_(inv_rm2sinthe2);
                const R diffusion_u = d2udr2 + (R)2.0 * u0 * G_(inv_rm2) + d2udthe2 * G_(inv_rm2) +
                                      (R)4.0 * dudr * G_(inv_rm) + dudthe * G_(costhe_inv_rm2sinthe) +
                                      d2udphi2 * G_(inv_rm2sinthe2);
                const R diffusion_v = d2vdr2 + dvdr * two_inv_rm + d2vdthe2 * G_(inv_rm2) +
                                      dvdthe * G_(costhe_inv_rm2sinthe) - G_(v_metric) * v0 +
                                      d2vdphi2 * G_(inv_rm2sinthe2) + (R)2.0 * dudthe * G_(inv_rm2) -
                                      dwdphi * (R)2.0 * G_(costhe) * G_(inv_rm2sinthe2);
                const R diffusion_w = d2wdr2 + dwdr * two_inv_rm + d2wdthe2 * G_(inv_rm2) +
                                      dwdthe * G_(costhe_inv_rm2sinthe) - G_(v_metric) * w0 +
                                      d2wdphi2 * G_(inv_rm2sinthe2) + (R)2.0 * dudphi * G_(inv_rm2sinthe) +
                                      dvdphi * (R)2.0 * G_(costhe) * G_(inv_rm2sinthe2);
#undef G_

                const R dpdr_term = (R)q.pgrad_scale * dpdr;
                const R dpdthe_term = (R)q.pgrad_scale * dpdthe * (R)g.inv_rm;
                const R dpdphi_term = (R)q.pgrad_scale * dpdphi * (R)g.inv_rmsinthe;
                R dphdthe_term = (R)0.0, dphdphi_term = (R)0.0;
                if (q.use_hp) {
                    const double hc = Ht[hP];
                    const double hjp = (wall && (nbm & NB_JP)) ? hc : Ht[hP + WP];
                    const double hjm = (wall && (nbm & NB_JM)) ? hc : Ht[hP - WP];
                    const double hkp = (wall && (nbm & NB_KP)) ? hc : Ht[hP + 1];
                    const double hkm = (wall && (nbm & NB_KM)) ? hc : Ht[hP - 1];
                    dphdthe_term = (R)((hjp - hjm) * q.inv_2dthe) * (R)g.inv_rm;
                    dphdphi_term = (R)((hkp - hkm) * q.inv_2dphi) * (R)g.inv_rmsinthe;
                }

                // radiative and latent heating (RHS_Jup_Turb.cpp:646-718)
                double radiation_t = 0.0, precip_t = 0.0;
                if (q.has_heating) {
                    if (q.rad_coupling != 0.0) {
                        const double T_phys = (double)t0 * q.t_ref;
                        const double P_phys = S.ps[cs][tid] * 1.0e5;
                        const double rho = (rho_l > 0.0 && isfinite(rho_l))
                                               ? rho_l
                                               : ((T_phys > 1.0) ? P_phys / (q.R_mix * T_phys) : 0.0);
                        if (rho > 0.0 && q.cp_mix > 0.0) {
                            radiation_t = q.rad_coupling * S.ex[xs][3][tid] * q.L_rad /
                                          (rho * q.cp_mix * q.u_0 * q.t_ref);
                            if (!isfinite(radiation_t)) radiation_t = 0.0;
                            else if (radiation_t > 0.5) radiation_t = 0.5;
                            else if (radiation_t < -0.5) radiation_t = -0.5;
                        }
                    }
                    if (q.precip_coupling != 0.0) {
                        double rho_p = q.r_mix;
                        if (q.precip_local) rho_p = (rho_l > 0.0 && isfinite(rho_l)) ? rho_l : q.r_mix;
                        if (rho_p > 0.0 && q.cp_mix > 0.0) {
                            precip_t = q.precip_coupling * S.ex[xs][4][tid] * q.L_rad /
                                       (rho_p * q.cp_mix * q.u_0 * q.t_ref);
                            if (!isfinite(precip_t)) precip_t = 0.0;
                            else if (precip_t > 0.5) precip_t = 0.5;
                            else if (precip_t < -0.5) precip_t = -0.5;
                        }
                    }
                }

                double nue_t = 0.0;
                if (q.has_nue) {
                    const double nn = S.ex[xs][2][tid];
                    if (q.turb_coupling != 0.0 && isfinite(nn)) nue_t = q.turb_coupling * fmax(0.0, nn);
                }
                const double nue_t_s = nue_t / 0.9;
                const R visc = (R)(q.inv_re + nue_t + S.ex[xs][1][tid]);

                const R rhs_t = +pressure_t - transport_t + diffusion_t * (R)(q.t_visc + nue_t_s) +
                                (R)radiation_t + (R)precip_t;
                // the buoyancy anomaly against the level mean, in FP64 (the mean is FP64)
                const double t0d = (double)t0;
                const double buoyancy_u =
                    (t0d > 0.0) ? q.buoy_k * (q.g * S.ps[cs][tid] / (q.rR * t0d * q.t_ref) - a.buoy_ref[i])
                                : 0.0;
                const R rhs_u = -dpdr_term + (q.hydro_split ? (R)0.0 : (R)buoyancy_u) - transport_u +
                                diffusion_u * visc - (R)(q.cor_rad_on * q.Coriolis) * Coriolis_rad +
                                (R)(q.centrifugal * g.cent_rad);
                const R rhs_v = -dpdthe_term - dphdthe_term - transport_v + diffusion_v * visc -
                                (R)q.Coriolis * Coriolis_the + (R)(q.centrifugal * g.cent_the);
                const R rhs_w = -dpdphi_term - dphdphi_term - transport_w + diffusion_w * visc -
                                (R)q.Coriolis * Coriolis_phi;

                // accumulate (RungeKutta_Jup_Turb.cpp:419-490), form the next stage input / result
                const R rhs[4] = {rhs_t, rhs_u, rhs_v, rhs_w};
                if (q.stage == 0) {
                    const double y0[4] = {(double)Tt[hT], (double)Ut[hT], (double)Vt[hT], (double)Wt[hT]};
#pragma unroll
                    for (int f = 0; f < 4; f++) {
                        if (!q.acc_free) static_cast<TA*>(a.acc[f])[c] = (TA)((R)q.wgt * rhs[f]);
                        static_cast<TO*>(a.Xo[f])[c] = (TO)(y0[f] + q.c_in * (double)rhs[f]);
                    }
                } else if (q.acc_free && q.stage < 3) {
                    // acc_free (FP64): stage 1 only forms X2; stage 2 forms X3 and the accumulator
                    // k1 + 2 k2 + 2 k3 with k1 = (X1 - y_n) / c, k2 = (X2 - y_n) / c
                    const double x2[4] = {(double)Tt[hT], (double)Ut[hT], (double)Vt[hT], (double)Wt[hT]};
#pragma unroll
                    for (int f = 0; f < 4; f++) {
                        const double yn = S.Yx[xs][f][tid];
                        if (q.stage == 2) {
                            const double k1 = ((double)S.ax[xs][f][tid] - yn) * q.inv_c_half;
                            const double k2 = (x2[f] - yn) * q.inv_c_half;
                            static_cast<TA*>(a.acc[f])[c] = (TA)((k1 + 2.0 * k2) + q.wgt * (double)rhs[f]);
                        }
                        static_cast<TO*>(a.Xo[f])[c] = (TO)(yn + q.c_in * (double)rhs[f]);
                    }
                } else if (q.stage < 3) {
#pragma unroll
                    for (int f = 0; f < 4; f++) {
                        static_cast<TA*>(a.acc[f])[c] = (TA)((R)S.ax[xs][f][tid] + (R)q.wgt * rhs[f]);
                        static_cast<TO*>(a.Xo[f])[c] = (TO)(S.Yx[xs][f][tid] + q.c_in * (double)rhs[f]);
                    }
                } else {
#pragma unroll
                    for (int f = 0; f < 4; f++) {
                        const double acc3 = (double)S.ax[xs][f][tid] + q.wgt * (double)rhs[f];
                        a.Y[f][c] = S.Yx[xs][f][tid] + q.dt * acc3 * q.one_sixth;
                    }
                    // the projection source the next pressure solve reads (the last stage's values)
                    a.aux_u[c] = (double)rhs_u + (double)dpdr_term;
                    a.aux_v[c] = (double)rhs_v + (double)dpdthe_term;
                    a.aux_w[c] = (double)rhs_w + (double)dpdphi_term;
                }
            }
        }
        if (live) {   // slide the radial window up one plane
            m_t = (double)Tt[hT]; m_u = (double)Ut[hT]; m_v = (double)Vt[hT]; m_w = (double)Wt[hT];
            m_pd = Pt[hP];
            m_ps = S.ps[cs][tid];
        }
        __syncthreads();
    }
}

// ---- buoyancy level mean (RungeKutta_Jup_Turb.cpp:47-69): fixed-order two-level reduction
constexpr int BR_BLOCKS = 16, BR_THREADS = 256;

__global__ void __launch_bounds__(BR_THREADS)
buoy_partial_kernel(const double* __restrict__ t, const double* __restrict__ p_stat,
                    const uint8_t* __restrict__ solid, const double* __restrict__ sin_the,
                    double* __restrict__ part, int jm, int km, int KP, double g, double rR,
                    double t_ref) {
    const int i = blockIdx.y, b = blockIdx.x;
    double s = 0.0, ws = 0.0;
    for (int j = b; j < jm; j += BR_BLOCKS) {
        const double wgt = sin_the[j];
        const size_t row = ((size_t)i * jm + j) * KP;
        for (int k = threadIdx.x; k < km; k += BR_THREADS) {
            if (solid[row + k]) continue;
            const double tt = t[row + k];
            if (!(tt > 0.0)) continue;
            const double bb = g * p_stat[row + k] / (rR * tt * t_ref);
            if (!isfinite(bb)) continue;
            s += wgt * bb;
            ws += wgt;
        }
    }
    __shared__ double sh_s[BR_THREADS / 32], sh_w[BR_THREADS / 32];
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
        ws += __shfl_down_sync(0xffffffffu, ws, o);
    }
    if ((threadIdx.x & 31) == 0) { sh_s[threadIdx.x >> 5] = s; sh_w[threadIdx.x >> 5] = ws; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ts = 0.0, tw = 0.0;
        for (int q = 0; q < BR_THREADS / 32; q++) { ts += sh_s[q]; tw += sh_w[q]; }
        part[(i * BR_BLOCKS + b) * 2 + 0] = ts;
        part[(i * BR_BLOCKS + b) * 2 + 1] = tw;
    }
}

__global__ void buoy_final_kernel(const double* __restrict__ part, double* __restrict__ out, int im) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= im) return;
    double s = 0.0, ws = 0.0;
    for (int b = 0; b < BR_BLOCKS; b++) {
        s += part[(i * BR_BLOCKS + b) * 2 + 0];
        ws += part[(i * BR_BLOCKS + b) * 2 + 1];
    }
    out[i] = (ws > 0.0) ? s / ws : 0.0;
}

// ---- hydrostatic pressure (RungeKutta_Jup_Turb.cpp:119-259), one thread per column.
// metric/Coriolis branch: f(i) = (v^2 + w^2) / r + cor * w over the fluid run [i0, i1] from
// zero at its foot, plus the frozen p_baro; solid cells below and cells above the run are 0.
__global__ void hydrostatic_kernel(const double* __restrict__ v, const double* __restrict__ w,
                                   const double* __restrict__ p_baro,
                                   const uint8_t* __restrict__ solid,
                                   const double* __restrict__ rad,
                                   const double* __restrict__ cor_col, double* __restrict__ ph,
                                   int im, int jm, int km, int KP, double dr) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (k >= km) return;
    const size_t plane = (size_t)jm * KP;
    const size_t base = (size_t)j * KP + k;
    int i0 = 0;
    while (i0 < im && solid[base + i0 * plane]) { ph[base + i0 * plane] = 0.0; i0++; }
    if (i0 >= im) return;
    int i1 = i0;
    while (i1 + 1 < im && !solid[base + (i1 + 1) * plane]) i1++;
    for (int i = i1 + 1; i < im; i++) ph[base + i * plane] = 0.0;
    const double cor = cor_col[j];
    double acc = 0.0, fprev = 0.0;
    for (int i = i0; i <= i1; i++) {
        const size_t c = base + i * plane;
        const double vv = v[c], ww = w[c];
        const double f = 0.0 + ((vv * vv + ww * ww) / rad[i] + cor * ww) / 1.0;
        if (i > i0) acc = acc + 0.5 * (fprev + f) * dr;
        fprev = f;
        ph[c] = acc + (p_baro ? p_baro[c] : 0.0);
    }
}

__global__ void mixture_density_kernel(const double* __restrict__ t, const double* __restrict__ ps,
                                       const double* __restrict__ pd, double* __restrict__ rho,
                                       size_t NP, double t_ref, double pdyn_w, double to_bar,
                                       double R_mix) {
    const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= NP) return;
    const double T = t[c] * t_ref;
    if (!(T > 0.0)) { rho[c] = 0.0; return; }
    const double p_pa = (ps[c] + pdyn_w * pd[c] * to_bar) * 1.0e5;
    const double r = p_pa / (R_mix * T);
    rho[c] = isfinite(r) ? r : 0.0;
}

}  // namespace

int launch_buoy_ref(AtjupCtx* c, const double* t) {
    const AtjupParams& P = c->P;
    dim3 grid(BR_BLOCKS, P.im);
    c->launches++;
    buoy_partial_kernel<<<grid, BR_THREADS, 0, c->stream>>>(
        t, c->f[ATJUP_F_P_STAT], c->solid, c->sin_the, c->red, P.jm, P.km, c->KP, P.g,
        P.r_mix * P.R_mix, P.t_ref);
    c->launches++;
    buoy_final_kernel<<<1, 64, 0, c->stream>>>(c->red, c->buoy_ref, P.im);
    ATJUP_CHECK_LAUNCH("buoy_ref");
    return ATJUP_OK;
}

int launch_hydrostatic(AtjupCtx* c, const double* v, const double* w) {
    const AtjupParams& P = c->P;
    if (!P.metric_split || P.hydro_split) {
        set_error("hydrostatic pressure: only the ATJUP_METRIC_SPLIT=1, ATJUP_HYDRO_SPLIT=0 form is implemented");
        return ATJUP_ERR_UNSUPPORTED;
    }
    dim3 grid((P.km + 127) / 128, P.jm);
    c->launches++;
    hydrostatic_kernel<<<grid, 128, 0, c->stream>>>(v, w, c->f[ATJUP_F_P_BARO], c->solid, c->rad,
                                                   c->cor_col, c->f[ATJUP_F_P_HYDRO], P.im, P.jm,
                                                   P.km, c->KP, P.dr);
    ATJUP_CHECK_LAUNCH("hydrostatic");
    return ATJUP_OK;
}

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime (the library does not
// link against the driver library)
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                 const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                 const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiled encode_tiled() {
    static EncodeTiled fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult qr{};
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault,
                                             &qr) == cudaSuccess &&
            qr == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(p);
        else
            cudaGetLastError();
    }
    return fn;
}

// a [im][jm][KP] array of T as a 3-D tensor (x = k, y = j, z = i) read in boxes of bw x bh x 1
// (halo boxes Box3<T>::W x HJ, cell boxes TK x TJ); the rows (KP T) and planes are multiples of
// 16 bytes
template <typename T>
static int make_box_map(CUtensorMap* m, const void* base, const AtjupCtx* c, int bw = Box3<T>::W,
                        int bh = HJ) {
    const EncodeTiled enc = encode_tiled();
    if (!enc) {
        set_error("rk_stage: cuTensorMapEncodeTiled is not available");
        return ATJUP_ERR_CUDA;
    }
    if (!base || reinterpret_cast<uintptr_t>(base) % 16) {
        set_error("rk_stage: a stage buffer is null or not 16-byte aligned");
        return ATJUP_ERR_ARG;
    }
    const AtjupParams& P = c->P;
    const cuuint64_t dim[3] = {(cuuint64_t)c->KP, (cuuint64_t)P.jm, (cuuint64_t)P.im};
    const cuuint64_t stride[2] = {(cuuint64_t)c->KP * sizeof(T), (cuuint64_t)P.jm * c->KP * sizeof(T)};
    const cuuint32_t box[3] = {(cuuint32_t)bw, (cuuint32_t)bh, 1u};
    const cuuint32_t estr[3] = {1u, 1u, 1u};
    const CUresult r = enc(m, sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                           3u, const_cast<void*>(base), dim, stride, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("rk_stage: cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
        return ATJUP_ERR_CUDA;
    }
    return ATJUP_OK;
}

template <typename TI, typename TO, typename TA, typename R>
static int launch_stage_t(AtjupCtx* c, const StagePtrs& a, const StageConst& q, const char* name) {
    const AtjupParams& P = c->P;
    static bool attr_set = false;       // one flag per instantiation
    if (!attr_set) {
        ATJUP_CUDA(cudaFuncSetAttribute(rk_stage_kernel<TI, TO, TA, R>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)sizeof(StageSmem<TI, TA>)));
        attr_set = true;
    }
    StageMaps M;
    memset(&M, 0, sizeof M);
    for (int f = 0; f < 4; f++)
        if (int rc = make_box_map<TI>(&M.x[f], a.X[f], c)) return rc;
    if (int rc = make_box_map<double>(&M.p[0], a.p_dyn, c)) return rc;
    if (int rc = make_box_map<double>(&M.p[1], a.p_hydro, c)) return rc;
    // the per-cell inputs the stage reads (issue_cells reads the same conditions)
    if (int rc = make_box_map<double>(&M.ps, a.p_stat, c, TK, TJ)) return rc;
    const double* ex[NX] = {a.rho, a.wall_nue, a.nue, a.Q_rad, a.Q_precip};
    for (int e = 0; e < NX; e++) {
        if ((e == 2 && !q.has_nue) || (e >= 3 && !q.has_heating)) continue;
        if (int rc = make_box_map<double>(&M.ex[e], ex[e], c, TK, TJ)) return rc;
    }
    if (q.stage > 0) {
        const bool need_ax = !q.acc_free || q.stage >= 2;
        const void* const* src = (q.acc_free && q.stage == 2) ? a.X1 : (const void* const*)a.acc;
        for (int f = 0; f < 4; f++) {
            if (int rc = make_box_map<double>(&M.y[f], a.Y[f], c, TK, TJ)) return rc;
            if (need_ax)
                if (int rc = make_box_map<TA>(&M.ax[f], src[f], c, TK, TJ)) return rc;
        }
    }
    dim3 grid((P.km - 1 + TK - 1) / TK, (P.jm + TJ - 1) / TJ, NCH);
    c->launches++;
    rk_stage_kernel<TI, TO, TA, R><<<grid, NT, sizeof(StageSmem<TI, TA>), c->stream>>>(a, q, M);
    ATJUP_CHECK_LAUNCH(name);
    return ATJUP_OK;
}

// Xin / Xout: the stage input and the next stage input (stage 0 reads the FP64 state itself;
// the other buffers are FP64 or, in the mixed step, FP32); X1: the stage-1 input, which stage 2
// reads in the FP64 step (may be null otherwise)
int launch_rk_stage(AtjupCtx* c, int stage, const void* const* Xin, void* const* Xout,
                    const void* const* X1) {
    const AtjupParams& P = c->P;
    StagePtrs a{};
    for (int f = 0; f < 4; f++) {
        a.X[f] = Xin[f];
        a.X1[f] = X1 ? X1[f] : nullptr;
        a.Xo[f] = Xout ? Xout[f] : nullptr;
        a.Y[f] = c->f[ATJUP_F_T + f];
        a.acc[f] = c->acc[f];
    }
    a.p_dyn = c->f[ATJUP_F_P_DYN];
    a.p_hydro = c->f[ATJUP_F_P_HYDRO];
    a.p_stat = c->f[ATJUP_F_P_STAT];
    a.rho = c->f[ATJUP_F_RHO_MIX];
    a.wall_nue = c->f[ATJUP_F_WALL_NUE];
    a.nue = c->f[ATJUP_F_NUE];
    a.Q_rad = c->f[ATJUP_F_Q_RAD];
    a.Q_precip = c->f[ATJUP_F_Q_PRECIP];
    a.aux_u = c->f[ATJUP_F_AUX_U];
    a.aux_v = c->f[ATJUP_F_AUX_V];
    a.aux_w = c->f[ATJUP_F_AUX_W];
    a.nb = c->nbflags;
    a.geo = c->geo;
    a.buoy_ref = c->buoy_ref;
    a.cell_vbar0 = c->cell_vbar0;
    a.cell_ubar0 = c->cell_ubar0;

    StageConst q{};
    q.im = P.im; q.jm = P.jm; q.km = P.km; q.KP = c->KP;
    q.stage = stage;
    q.c_in = (stage == 0 || stage == 1) ? 0.5 * P.dt : (stage == 2 ? P.dt : 0.0);
    q.wgt = (stage == 0 || stage == 3) ? 1.0 : 2.0;
    q.dt = P.dt;
    q.one_sixth = 1.0 / 6.0;
    q.inv_2dr = 1.0 / (2.0 * P.dr);
    q.inv_2dthe = 1.0 / (2.0 * P.dthe);
    q.inv_2dphi = 1.0 / (2.0 * P.dphi);
    q.inv_dr2 = 1.0 / (P.dr * P.dr);
    q.inv_dthe2 = 1.0 / (P.dthe * P.dthe);
    q.inv_dphi2 = 1.0 / (P.dphi * P.dphi);
    q.cor_phi_f = P.nd_cor * +2.0 * P.omega;
    q.coeff_energy_p = P.u_0 * P.u_0 / (P.cp_mix * P.t_ref);
    q.to_nd = 1.0 / P.p_dyn_to_bar;
    q.r_mix = P.r_mix;
    q.rR = P.r_mix * P.R_mix;
    q.g = P.g;
    q.t_ref = P.t_ref;
    q.R_mix = P.R_mix;
    q.cp_mix = P.cp_mix;
    q.u_0 = P.u_0;
    q.L_rad = P.L_atm * 1.0e3;
    q.t_visc = P.t_diff_scale / (P.re * P.pr);
    q.inv_re = 1.0 / P.re;
    q.buoy_k = -P.nd_buoy * P.buoy_scale * P.buoy_ramp * P.buoyancy;
    q.metric_on = P.metric_split ? 0.0 : 1.0;
    q.cor_rad_on = P.coriolis_split ? 0.0 : 1.0;
    q.Coriolis = P.Coriolis;
    q.centrifugal = P.centrifugal;
    q.pgrad_scale = P.pgrad_scale;
    q.rad_coupling = P.rad_coupling;
    q.precip_coupling = P.precip_coupling;
    q.turb_coupling = P.turb_coupling;
    q.pgrad_wall = P.pgrad_wall;
    q.adiabatic = P.adiabatic;
    q.adiabatic_rho = P.adiabatic_rho;
    q.hydro_split = P.hydro_split;
    q.use_hp = (P.hydro_split || P.metric_split) ? 1 : 0;
    q.cell_hold = (P.cell_hold && c->cell_vbar0) ? 1 : 0;
    q.has_nue = (P.has_nue && a.nue) ? 1 : 0;
    q.has_heating = (P.has_heating && a.Q_rad && a.Q_precip) ? 1 : 0;
    q.precip_local = (P.precip_rho_local && P.local_rho) ? 1 : 0;
    q.acc_free = (c->step_prec != ATJUP_PREC_MIXED) ? 1 : 0;
    q.inv_c_half = 2.0 / P.dt;
    if (q.acc_free && stage == 2 && !X1) {
        set_error("rk_stage: stage 2 needs the stage-1 input");
        return ATJUP_ERR_ARG;
    }

    if (c->step_prec != ATJUP_PREC_MIXED)
        return launch_stage_t<double, double, double, double>(c, a, q, "rk_stage");
    if (stage == 0) return launch_stage_t<double, float, float, float>(c, a, q, "rk_stage (mixed)");
    return launch_stage_t<float, float, float, float>(c, a, q, "rk_stage (mixed)");
}

int launch_mixture_density(AtjupCtx* c) {
    const AtjupParams& P = c->P;
    const int th = 256;
    const size_t nb = (c->NP + th - 1) / th;
    c->launches++;
    mixture_density_kernel<<<(unsigned)nb, th, 0, c->stream>>>(
        c->f[ATJUP_F_T], c->f[ATJUP_F_P_STAT], c->f[ATJUP_F_P_DYN], c->f[ATJUP_F_RHO_MIX], c->NP,
        P.t_ref, P.rho_pdyn ? 1.0 : 0.0, P.p_dyn_to_bar, P.R_mix);
    ATJUP_CHECK_LAUNCH("mixture_density");
    return ATJUP_OK;
}

}  // namespace atjup
