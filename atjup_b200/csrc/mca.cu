// Moist convective adjustment with the Ledoux criterion, per column.
//
// Reference: MoistConvectiveAdjustment<cJupiterModel>::run (ConvectiveAdjustment.h:403-849), called
// by the loop after the boundary passes (cJupiterModel.cpp:1300-1320) with the gases H2O and NH3
// and the tracers H2S, NH4SH (and the chromophore, zero unless ATJUP_CHROM is on). Jupiter's
// defaults: no latitude smoothing, the t_0 phase rule, constant cp.
//
// Each column is swept bottom-up; a pair (a, a+1) is unstable when a parcel lifted from a to a+1,
// conserving h_L = cp T + g z - sum(lv q_liq + ls q_ice) - L_NH4SH q_NH4SH and the total of every
// gas, is lighter (higher virtual temperature) than the air at a+1 in its own equilibrium. An
// unstable segment is mixed (mass-weighted h_L, q_t, tracers) and settled back to equilibrium,
// grows while its edges are unstable, and sweeps repeat. In practice almost every column is
// stable, and deciding that is the cost: every pair needs two equilibrium solves. So the work is
// split:
//   mca_census_kernel   one thread per pair (i, i+1) of every column: the reference's census of
//                       the unadjusted column (the pair test, the "held by composition" count);
//                       a column with an unstable pair, or with a cell the reference would refuse,
//                       is appended to a list.
//   mca_column_kernel   one thread per listed column: the reference's whole column algorithm
//                       (starting from the census the census kernel recorded per pair, the sweeps,
//                       the segment growth, the relaxation, the write-back), with the column's
//                       state in a per-thread slot in global memory; with few listed columns
//   mca_column_warp_kernel  instead, one warp per column, its independent parts (the settles of a
//                       mixed segment, the pair tests of a sweep) on the lanes.
// A column that is not listed is left alone by the reference too (no unstable pair: pass 1 mixes
// nothing). The equilibrium solve and every expression keep the reference's operand order, and
// the file is compiled without FMA contraction; the parcel test compares a virtual-temperature
// difference with 1e-7 K, so a last-bit difference of exp/log can flip a marginal pair.
#include "ctx.cuh"

namespace atjup {
namespace {

constexpr int NG = 2, NT = 2;          // gases H2O, NH3; tracers H2S, NH4SH
constexpr int MAXI = 64;               // levels a column slot holds (the reference grid has 41)
constexpr int NITER = 60;              // cap of the equilibrium solve
constexpr double TOL_K = 1.0e-7, TOL_T = 1.0e-10;
constexpr int NSLOT = 4096;            // columns adjusted concurrently (scratch slots)
constexpr int NPART = 256;             // partial census counters (spread so the adds do not contend)

__device__ __forceinline__ double dmax(double a, double b) { return a < b ? b : a; }

struct McaArgs {
    double* t;
    const double *p_stat, *rho_mix;
    double* vap[NG];
    double* cld[NG];
    double* ice[NG];
    double* trf[NT];
    const uint8_t* solid;
    const float* layer_h;
    const int2* bounds;                // [jm * km] (i0, i1) of the column, interior applied
    AtjupGasParams gas[NG];
    double tr_ep[NT], tr_L[NT];
    int tr_cond[NT];
    double cp, grav, t_ref, r_mix, relax;
    int im, jm, km, KP, local_rho, ledoux, loading, max_pass;
    unsigned long long* stats;         // [8], then NPART pairs of census partial counts
    unsigned* colflag;                 // [jm * km]
    unsigned* list;                    // [jm * km] listed columns
    unsigned* count;
    uint8_t* pairs;                    // [im * jm * km] census of pair (i, i+1): bit 0 unstable, bit 1 moist
};

// ATPhys.h:49-52 [bar], with log(T) passed in: both gases are evaluated at the same T, and the
// logarithm (a pure function) is the same value whether computed once or per gas
__device__ __forceinline__ double svp(double T, double lT, double C, double L0, double R, double da,
                                      double db) {
    return exp(C + (-L0 / T + da * lT + db * T) / (1e-3 * R));
}
// the phase's coefficients are selected first, so the saturation curve is one exp in the code
// (the liquid and ice curves are the same expression on different constants)
__device__ __forceinline__ double qsat(const McaArgs& a, int g, double T, double lT, double p) {
    const AtjupGasParams& s = a.gas[g];
    const bool liq = T >= s.t_0;
    const double E = svp(T, lT, liq ? s.C : s.C_i, liq ? s.L0 : s.L0_i, s.R,
                         liq ? s.del_alf : s.del_alf_i, liq ? s.del_bet : s.del_bet_i);
    const double q = s.ep * E / p;
    return isfinite(q) ? q : 0.0;
}
__device__ __forceinline__ double lat(const McaArgs& a, int g, double T) {
    return T >= a.gas[g].t_0 ? a.gas[g].lv : a.gas[g].ls;
}
__device__ __forceinline__ double fof(const McaArgs& a, double TT, double hL, const double* qt,
                                      double p, double z) {
    double f = a.cp * TT + a.grav * z - hL;
    const double lT = log(TT);
    for (int g = 0; g < NG; g++) f -= lat(a, g, TT) * dmax(0.0, qt[g] - qsat(a, g, TT, lT, p));
    return f;
}
// equilibrium temperature of (h_L, q_t) at (p, z): Illinois regula falsi in [all vapour, all
// condensed] (ConvectiveAdjustment.h:459-486)
__device__ bool equil(const McaArgs& a, double hL, const double* qt, double p, double z, double& T,
                      double* cond) {
    const double T_lo = (hL - a.grav * z) / a.cp;
    if (!(T_lo > 0.0) || !(p > 0.0)) return false;
    bool any = false;
    const double lT_lo = log(T_lo);
    for (int g = 0; g < NG; g++)
        if (qt[g] > qsat(a, g, T_lo, lT_lo, p)) { any = true; break; }
    if (!any) {
        T = T_lo;
        for (int g = 0; g < NG; g++) cond[g] = 0.0;
        return true;
    }
    double span = 0.0;
    for (int g = 0; g < NG; g++) span += dmax(a.gas[g].lv, a.gas[g].ls) * dmax(0.0, qt[g]);
    double lo = T_lo, hi = T_lo + span / a.cp + 1.0e-9;
    double flo = fof(a, lo, hL, qt, p, z), fhi = fof(a, hi, hL, qt, p, z);
    int side = 0;
    for (int it = 0; it < NITER && hi - lo > TOL_T; it++) {
        double c = (fhi - flo != 0.0) ? hi - fhi * (hi - lo) / (fhi - flo) : 0.5 * (lo + hi);
        if (!(c > lo && c < hi)) c = 0.5 * (lo + hi);
        const double fc = fof(a, c, hL, qt, p, z);
        if (fc < 0.0) { lo = c; flo = fc; if (side == -1) fhi *= 0.5; side = -1; }
        else          { hi = c; fhi = fc; if (side == +1) flo *= 0.5; side = +1; }
        if (fabs(fc) <= a.cp * TOL_T) { lo = hi = c; break; }
    }
    T = hi;
    const double lT = log(T);
    for (int g = 0; g < NG; g++) cond[g] = dmax(0.0, qt[g] - qsat(a, g, T, lT, p));
    return true;
}

// One cell's conserved state: mass fractions, h_L, and the inputs of the parcel test.
struct Cell {
    double T, p, z, rho, hL;
    double qt[NG], qv[NG], qc[NG], qi[NG], qr[NT];
};
// loads cell (i, j, k); false when the reference would refuse the column for it
__device__ bool load_cell(const McaArgs& a, int i, size_t c, Cell& x) {
    x.T = a.t[c] * a.t_ref;
    x.p = a.p_stat[c];
    x.z = (double)a.layer_h[i] * 1.0e3;
    double r = a.r_mix;
    if (a.local_rho) { const double rr = a.rho_mix[c]; r = (rr > 0.0 && isfinite(rr)) ? rr : a.r_mix; }
    x.rho = r;
    if (!(x.T > 0.0) || !(x.p > 0.0) || !(x.rho > 0.0) || !isfinite(x.T + x.p + x.rho)) return false;
    double h = a.cp * x.T + a.grav * x.z;
    for (int g = 0; g < NG; g++) {
        x.qv[g] = dmax(0.0, a.vap[g][c]) / x.rho;
        x.qc[g] = dmax(0.0, a.cld[g][c]) / x.rho;
        x.qi[g] = dmax(0.0, a.ice[g][c]) / x.rho;
        x.qt[g] = x.qv[g] + x.qc[g] + x.qi[g];
        h -= a.gas[g].lv * x.qc[g] + a.gas[g].ls * x.qi[g];
    }
    for (int r2 = 0; r2 < NT; r2++) {
        x.qr[r2] = a.trf[r2][c] / x.rho;
        h -= a.tr_L[r2] * x.qr[r2];
    }
    x.hL = h;
    return true;
}
__device__ __forceinline__ double trE(const McaArgs& a, const double* qr) {
    double e = 0.0;
    for (int r = 0; r < NT; r++) e += a.tr_L[r] * qr[r];
    return e;
}
__device__ __forceinline__ double tv(const McaArgs& a, double TT, const double* v,
                                     const double* cnd, const double* qr) {
    if (!a.ledoux) return TT;
    double f = 1.0;
    for (int g = 0; g < NG; g++) {
        f += v[g] * (1.0 / a.gas[g].ep - 1.0);
        if (a.loading) f -= cnd[g];
    }
    for (int r = 0; r < NT; r++) {
        const double q = qr[r];
        if (a.tr_ep[r] > 0.0) f += q * (1.0 / a.tr_ep[r] - 1.0);
        else if (a.tr_cond[r] && a.loading) f -= q;
    }
    return TT * f;
}
// the parcel test of a below b (ConvectiveAdjustment.h:651-665) given b's own equilibrium
__device__ bool pair_test(const McaArgs& a, double hLa, const double* qta, const double* qra,
                          double pb, double zb, double Tb, const double* ecb, const double* qtb,
                          const double* qrb, bool& ok, bool* held, bool* moist) {
    double Tp, pc[NG], pv[NG], ev[NG];
    ok = equil(a, hLa + trE(a, qra), qta, pb, zb, Tp, pc);
    if (!ok) return false;
    bool wet = false;
    for (int g = 0; g < NG; g++) {
        pv[g] = qta[g] - pc[g];
        if (pc[g] > 0.0) wet = true;
        ev[g] = qtb[g] - ecb[g];
    }
    const double dTv = tv(a, Tp, pv, pc, qra) - tv(a, Tb, ev, ecb, qrb);
    if (held) *held = (Tp - Tb > TOL_K) && !(dTv > TOL_K);
    if (moist) *moist = wet;
    return dTv > TOL_K;
}

__device__ __forceinline__ void enqueue(const McaArgs& a, unsigned col) {
    if (atomicExch(&a.colflag[col], 1u) == 0u) a.list[atomicAdd(a.count, 1u)] = col;
}

// (i0, i1) of every column from the static mask (ConvectiveAdjustment.h:527-540)
__global__ void mca_bounds_kernel(const uint8_t* solid, int2* bounds, int im, int jm, int km,
                                  int KP, int interior) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (k >= km) return;
    const size_t plane = (size_t)jm * KP, c0 = (size_t)j * KP + k;
    int i0 = 0;
    while (i0 < im && solid[c0 + (size_t)i0 * plane] == 1) i0++;
    int i1 = i0;
    while (i1 + 1 < im && solid[c0 + (size_t)(i1 + 1) * plane] != 1) i1++;
    if (interior) { if (i0 == 0) i0 = 1; if (i1 == im - 1) i1 = im - 2; }
    bounds[(size_t)j * km + k] = make_int2(i0, i1);
}

// one thread per pair (i, i+1): the census of the unadjusted column. Capped at 64 registers
// (eight blocks per SM): the solve is a chain of dependent FP64 exp/log, and the extra warps hide
// more of it than the few spilled values cost.
__global__ void __launch_bounds__(128, 8) mca_census_kernel(McaArgs a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, i = blockIdx.z;
    unsigned long long ut = 0, hd = 0;
    if (k < a.km) {
        const int2 b = a.bounds[(size_t)j * a.km + k];
        if (b.y - b.x >= 1 && i >= b.x && i < b.y) {
            const unsigned col = (unsigned)(j * a.km + k);
            const size_t plane = (size_t)a.jm * a.KP, c = (size_t)j * a.KP + k + (size_t)i * plane;
            Cell lo, up;
            const bool v0 = load_cell(a, i, c, lo), v1 = load_cell(a, i + 1, c + plane, up);
            if (!v0 || !v1) {
                enqueue(a, col);       // the column thread counts it as skipped
            } else {
                double Tb, ecb[NG];
                bool ok = equil(a, up.hL + trE(a, up.qr), up.qt, up.p, up.z, Tb, ecb);
                bool held = false, moist = false, uns = false;
                if (ok) uns = pair_test(a, lo.hL, lo.qt, lo.qr, up.p, up.z, Tb, ecb, up.qt, up.qr, ok, &held, &moist);
                if (uns || held) ut = 1;
                if (held) hd = 1;
                a.pairs[((size_t)i * a.jm + j) * a.km + k] = (uint8_t)((uns ? 1 : 0) | (moist ? 2 : 0));
                if (uns) enqueue(a, col);
            }
        }
    }
    // the census counters: a warp sum, added by lane 0 to one of NPART partial counters (summed on
    // the host). No block barrier: a warp whose pairs took no iterative solve leaves at once
    // instead of waiting for the slowest warp of its block, and the partials keep the adds from
    // contending on one address.
    for (int o = 16; o > 0; o >>= 1) {
        ut += __shfl_down_sync(0xffffffffu, ut, o);
        hd += __shfl_down_sync(0xffffffffu, hd, o);
    }
    if ((threadIdx.x & 31) == 0 && (ut | hd)) {
        const unsigned warp = (blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)) *
                              (blockDim.x >> 5) + (threadIdx.x >> 5);
        const unsigned part = warp % NPART;
        if (ut) atomicAdd(&a.stats[8 + 2 * part], ut);
        if (hd) atomicAdd(&a.stats[9 + 2 * part], hd);
    }
}

// A column's state, one per scratch slot (ConvectiveAdjustment.h:546-645).
struct Col {
    double T[MAXI], p[MAXI], z[MAXI], rho[MAXI], w[MAXI], hL[MAXI], T0[MAXI], Teq[MAXI], hL0[MAXI];
    double qt[MAXI][NG], qv[MAXI][NG], qc[MAXI][NG], qi[MAXI][NG], ceq[MAXI][NG], qt0[MAXI][NG];
    double qr[MAXI][NT], qr0[MAXI][NT];
    char eq_ok[MAXI], touched[MAXI], cen_u[MAXI], cen_m[MAXI];
    char pt_u[MAXI];           // the pair tests of a sweep on the state it starts from
    char dirty[MAXI];          // mixed since those tests
};

__device__ bool col_unstable(const McaArgs& a, Col& C, int lo, int up, bool* held, bool* moist) {
    if (!C.eq_ok[up]) {
        if (!equil(a, C.hL[up] + trE(a, C.qr[up]), C.qt[up], C.p[up], C.z[up], C.Teq[up], C.ceq[up]))
            return false;
        C.eq_ok[up] = 1;
    }
    // the reference solves the parcel before the cached air state; both are pure functions
    bool ok;
    return pair_test(a, C.hL[lo], C.qt[lo], C.qr[lo], C.p[up], C.z[up], C.Teq[up], C.ceq[up],
                     C.qt[up], C.qr[up], ok, held, moist);
}
__device__ bool col_settle(const McaArgs& a, Col& C, int q) {
    double TT, pc[NG];
    if (!equil(a, C.hL[q] + trE(a, C.qr[q]), C.qt[q], C.p[q], C.z[q], TT, pc)) return false;
    C.T[q] = TT;
    C.Teq[q] = TT;
    C.eq_ok[q] = 1;
    for (int g = 0; g < NG; g++) {
        C.ceq[q][g] = pc[g];
        C.qv[q][g] = C.qt[q][g] - pc[g];
        if (TT >= a.gas[g].t_0) { C.qc[q][g] = pc[g]; C.qi[q][g] = 0.0; }
        else { C.qi[q][g] = pc[g]; C.qc[q][g] = 0.0; }
    }
    C.touched[q] = 1;
    return true;
}
__device__ bool col_mix(const McaArgs& a, Col& C, int lo, int up) {
    double sw = 0.0, sh = 0.0, sq[NG] = {0.0, 0.0}, sr[NT] = {0.0, 0.0};
    for (int q = lo; q <= up; q++) {
        sw += C.w[q];
        sh += C.w[q] * C.hL[q];
        for (int g = 0; g < NG; g++) sq[g] += C.w[q] * C.qt[q][g];
        for (int r = 0; r < NT; r++) sr[r] += C.w[q] * C.qr[q][r];
    }
    for (int q = lo; q <= up; q++) {
        C.hL[q] = sh / sw;
        for (int g = 0; g < NG; g++) C.qt[q][g] = sq[g] / sw;
        for (int r = 0; r < NT; r++) C.qr[q][r] = sr[r] / sw;
        if (!col_settle(a, C, q)) return false;
    }
    return true;
}

// Many listed columns (more than WARP_COLS_MAX): one thread per listed column, NSLOT threads in
// blocks of COL_BLOCK; listed column idx goes to lane idx / blocks of block idx % blocks. The
// lanes of a warp then walk 32 columns at once, which keeps the FP64 units busier than a warp's
// lone walk (measured: 5,910 columns with ~23 mixed layers each, 10.6 ms against 19.2 ms one
// warp per column). With few columns a warp per column is faster (1,562 columns of single-pair
// mixes: 0.24 ms against 0.86 ms): mca_column_warp_kernel. Both give the same bits.
constexpr int COL_BLOCK = 32;
constexpr unsigned WARP_COLS_MAX = 2048;
__global__ void __launch_bounds__(COL_BLOCK) mca_column_kernel(McaArgs a, Col* slots) {
    const unsigned slot = blockIdx.x * blockDim.x + threadIdx.x;
    Col& C = slots[slot];
    const unsigned n = *a.count;
    if (n <= WARP_COLS_MAX) return;
    for (unsigned idx = threadIdx.x * gridDim.x + blockIdx.x; idx < n; idx += NSLOT) {
        const unsigned col = a.list[idx];
        const int j = (int)(col / (unsigned)a.km), k = (int)(col % (unsigned)a.km);
        const int2 b = a.bounds[col];
        const int i0 = b.x, i1 = b.y;
        const size_t plane = (size_t)a.jm * a.KP, c0 = (size_t)j * a.KP + k;
        bool ok = true;
        for (int i = i0; i <= i1; i++) { C.eq_ok[i] = 0; C.touched[i] = 0; }
        for (int i = i0; i <= i1 && ok; i++) {
            Cell x;
            ok = load_cell(a, i, c0 + (size_t)i * plane, x);
            if (!ok) break;
            C.T[i] = C.T0[i] = x.T;
            C.p[i] = x.p;
            C.z[i] = x.z;
            C.rho[i] = x.rho;
            C.hL[i] = x.hL;
            for (int g = 0; g < NG; g++) {
                C.qt[i][g] = x.qt[g]; C.qv[i][g] = x.qv[g]; C.qc[i][g] = x.qc[g]; C.qi[i][g] = x.qi[g];
            }
            for (int r = 0; r < NT; r++) C.qr[i][r] = x.qr[r];
        }
        if (ok)
            for (int i = i0; i <= i1 && ok; i++) {
                const double lo = (i > i0) ? 0.5 * (C.z[i - 1] + C.z[i]) : C.z[i0];
                const double hi = (i < i1) ? 0.5 * (C.z[i] + C.z[i + 1]) : C.z[i1];
                C.w[i] = C.rho[i] * (hi - lo);
                if (!(C.w[i] > 0.0)) ok = false;
            }
        if (!ok) { atomicAdd(&a.stats[6], 1ull); continue; }
        // the census of the first sweep, as the census kernel found it (the same pair tests on the
        // same state); every pair of a column that loads is written there
        for (int i = i0; i < i1; i++) {
            const uint8_t f = a.pairs[((size_t)i * a.jm + j) * a.km + k];
            C.cen_u[i] = f & 1;
            C.cen_m[i] = (f >> 1) & 1;
        }
        for (int i = i0; i <= i1; i++) {
            C.hL0[i] = C.hL[i];
            for (int g = 0; g < NG; g++) C.qt0[i][g] = C.qt[i][g];
            for (int r = 0; r < NT; r++) C.qr0[i][r] = C.qr[i][r];
        }
        int passes = 0;
        long long layers = 0, moist_t = 0, dry_t = 0;
        bool changed = true, fail = false;
        while (changed && passes < a.max_pass && !fail) {
            changed = false;
            passes++;
            int i = i0;
            while (i < i1 && !fail) {
                bool moist = false, uns;
                if (passes == 1 && !C.touched[i] && !C.touched[i + 1]) { uns = C.cen_u[i]; moist = C.cen_m[i]; }
                else uns = col_unstable(a, C, i, i + 1, nullptr, &moist);
                if (!uns) { i++; continue; }
                if (passes == 1) { if (moist) moist_t++; else dry_t++; }
                int lo = i, up = i + 1;
                for (;;) {
                    if (!col_mix(a, C, lo, up)) { fail = true; break; }
                    bool ext = false;
                    if (lo > i0 && col_unstable(a, C, lo - 1, lo, nullptr, nullptr)) { lo--; ext = true; }
                    if (up < i1 && col_unstable(a, C, up, up + 1, nullptr, nullptr)) { up++; ext = true; }
                    if (!ext) break;
                }
                layers += up - lo + 1;
                changed = true;
                i = up;
            }
        }
        if (passes >= 1 && (moist_t || dry_t)) {
            atomicAdd(&a.stats[2], (unsigned long long)moist_t);
            atomicAdd(&a.stats[3], (unsigned long long)dry_t);
        }
        if (fail) { atomicAdd(&a.stats[6], 1ull); continue; }
        if (layers == 0) continue;
        if (a.relax < 1.0) {
            for (int q = i0; q <= i1 && !fail; q++) {
                if (!C.touched[q]) continue;
                C.hL[q] = C.hL0[q] + a.relax * (C.hL[q] - C.hL0[q]);
                for (int g = 0; g < NG; g++) C.qt[q][g] = C.qt0[q][g] + a.relax * (C.qt[q][g] - C.qt0[q][g]);
                for (int r = 0; r < NT; r++) C.qr[q][r] = C.qr0[q][r] + a.relax * (C.qr[q][r] - C.qr0[q][r]);
                if (!col_settle(a, C, q)) fail = true;
            }
            if (fail) { atomicAdd(&a.stats[6], 1ull); continue; }
        }
        for (int q = i0; q <= i1; q++) {
            if (!C.touched[q]) continue;
            const size_t c = c0 + (size_t)q * plane;
            a.t[c] = C.T[q] / a.t_ref;
            for (int g = 0; g < NG; g++) {
                a.vap[g][c] = C.qv[q][g] * C.rho[q];
                a.cld[g][c] = C.qc[q][g] * C.rho[q];
                a.ice[g][c] = C.qi[q][g] * C.rho[q];
            }
            for (int r = 0; r < NT; r++) a.trf[r][c] = C.qr[q][r] * C.rho[q];
        }
        atomicAdd(&a.stats[0], 1ull);
        atomicAdd(&a.stats[1], (unsigned long long)layers);
        atomicMax(&a.stats[7], (unsigned long long)passes);
    }
}

// Few listed columns (at most WARP_COLS_MAX): one warp per listed column, NSLOT warps, COL_WARPS
// per block; listed column idx goes to warp idx / blocks of block idx % blocks. The
// reference's algorithm walks the column in order, but most of its work is independent: the
// loads, the settles of a mixed segment (one equilibrium solve per level), the two edge tests of
// a growing segment, and, from the second sweep on, the pair tests of the sweep on the state it
// starts from (a pair whose two levels no mix of the sweep has touched yet tests the same then as
// when the walk reaches it: the test is a pure function of the two levels). The lanes take those;
// the walk itself (the next pair, the segment's bounds, a mix's sums in the reference's order)
// runs in step on every lane, and a lone test on lane 0. Every value comes from the same
// expression as in the sequential algorithm, so the result is the same.
constexpr int COL_WARPS = 4;
constexpr unsigned FULL_WARP = 0xffffffffu;

// the pair test (lo, up) on lane 0 (it may fill the equilibrium cache of up), its result on every
// lane
__device__ bool warp_unstable(const McaArgs& a, Col& C, int lo, int up, bool* moist, unsigned lane) {
    int u = 0, m = 0;
    if (lane == 0) {
        bool mm = false;
        u = col_unstable(a, C, lo, up, nullptr, &mm) ? 1 : 0;
        m = mm ? 1 : 0;
    }
    __syncwarp();
    u = __shfl_sync(FULL_WARP, u, 0);
    m = __shfl_sync(FULL_WARP, m, 0);
    if (moist) *moist = m != 0;
    return u != 0;
}

// col_mix with the levels' settles spread over the lanes: the sums on every lane in the
// reference's order, then each lane sets and settles its levels. A failed settle abandons the
// column, so the levels set after it do not matter.
__device__ bool warp_mix(const McaArgs& a, Col& C, int lo, int up, unsigned lane) {
    double sw = 0.0, sh = 0.0, sq[NG] = {0.0, 0.0}, sr[NT] = {0.0, 0.0};
    for (int q = lo; q <= up; q++) {
        sw += C.w[q];
        sh += C.w[q] * C.hL[q];
        for (int g = 0; g < NG; g++) sq[g] += C.w[q] * C.qt[q][g];
        for (int r = 0; r < NT; r++) sr[r] += C.w[q] * C.qr[q][r];
    }
    __syncwarp();
    bool ok = true;
    for (int q = lo + (int)lane; q <= up; q += 32) {
        C.hL[q] = sh / sw;
        for (int g = 0; g < NG; g++) C.qt[q][g] = sq[g] / sw;
        for (int r = 0; r < NT; r++) C.qr[q][r] = sr[r] / sw;
        C.dirty[q] = 1;
        if (ok && !col_settle(a, C, q)) ok = false;
    }
    ok = __all_sync(FULL_WARP, ok) != 0;
    __syncwarp();
    return ok;
}

__global__ void __launch_bounds__(32 * COL_WARPS) mca_column_warp_kernel(McaArgs a, Col* slots) {
    const unsigned lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
    Col& C = slots[blockIdx.x * COL_WARPS + wi];
    const unsigned n = *a.count;
    if (n > WARP_COLS_MAX) return;
    for (unsigned idx = wi * gridDim.x + blockIdx.x; idx < n; idx += NSLOT) {
        const unsigned col = a.list[idx];
        const int j = (int)(col / (unsigned)a.km), k = (int)(col % (unsigned)a.km);
        const int2 b = a.bounds[col];
        const int i0 = b.x, i1 = b.y;
        const size_t plane = (size_t)a.jm * a.KP, c0 = (size_t)j * a.KP + k;
        // the column's cells (the reference refuses the whole column for any one of them)
        bool ok = true;
        for (int i = i0 + (int)lane; i <= i1; i += 32) {
            C.eq_ok[i] = 0;
            C.touched[i] = 0;
            C.dirty[i] = 0;
            Cell x;
            if (!load_cell(a, i, c0 + (size_t)i * plane, x)) { ok = false; continue; }
            C.T[i] = C.T0[i] = x.T;
            C.p[i] = x.p;
            C.z[i] = x.z;
            C.rho[i] = x.rho;
            C.hL[i] = x.hL;
            for (int g = 0; g < NG; g++) {
                C.qt[i][g] = x.qt[g]; C.qv[i][g] = x.qv[g]; C.qc[i][g] = x.qc[g]; C.qi[i][g] = x.qi[g];
            }
            for (int r = 0; r < NT; r++) C.qr[i][r] = x.qr[r];
        }
        ok = __all_sync(FULL_WARP, ok) != 0;
        __syncwarp();
        if (ok) {
            for (int i = i0 + (int)lane; i <= i1; i += 32) {
                const double lo = (i > i0) ? 0.5 * (C.z[i - 1] + C.z[i]) : C.z[i0];
                const double hi = (i < i1) ? 0.5 * (C.z[i] + C.z[i + 1]) : C.z[i1];
                C.w[i] = C.rho[i] * (hi - lo);
                if (!(C.w[i] > 0.0)) ok = false;
            }
            ok = __all_sync(FULL_WARP, ok) != 0;
        }
        if (!ok) {
            if (lane == 0) atomicAdd(&a.stats[6], 1ull);
            __syncwarp();
            continue;
        }
        // the census of the first sweep, as the census kernel found it (the same pair tests on the
        // same state); every pair of a column that loads is written there
        for (int i = i0 + (int)lane; i < i1; i += 32) {
            const uint8_t f = a.pairs[((size_t)i * a.jm + j) * a.km + k];
            C.cen_u[i] = f & 1;
            C.cen_m[i] = (f >> 1) & 1;
        }
        for (int i = i0 + (int)lane; i <= i1; i += 32) {
            C.hL0[i] = C.hL[i];
            for (int g = 0; g < NG; g++) C.qt0[i][g] = C.qt[i][g];
            for (int r = 0; r < NT; r++) C.qr0[i][r] = C.qr[i][r];
        }
        __syncwarp();
        int passes = 0;
        long long layers = 0, moist_t = 0, dry_t = 0;
        bool changed = true, fail = false;
        while (changed && passes < a.max_pass && !fail) {
            changed = false;
            passes++;
            if (passes >= 2) {
                for (int i = i0 + (int)lane; i < i1; i += 32) {
                    bool m = false;
                    C.pt_u[i] = col_unstable(a, C, i, i + 1, nullptr, &m) ? 1 : 0;
                }
                for (int i = i0 + (int)lane; i <= i1; i += 32) C.dirty[i] = 0;
                __syncwarp();
            }
            int i = i0;
            while (i < i1 && !fail) {
                bool moist = false, uns;
                if (passes == 1 && !C.touched[i] && !C.touched[i + 1]) { uns = C.cen_u[i]; moist = C.cen_m[i]; }
                else if (passes >= 2 && !C.dirty[i] && !C.dirty[i + 1]) uns = C.pt_u[i];
                else uns = warp_unstable(a, C, i, i + 1, &moist, lane);
                if (!uns) { i++; continue; }
                if (passes == 1) { if (moist) moist_t++; else dry_t++; }
                int lo = i, up = i + 1;
                for (;;) {
                    if (!warp_mix(a, C, lo, up, lane)) { fail = true; break; }
                    // the two edge tests, independent of each other, on lanes 0 and 1
                    int e0 = 0, e1 = 0;
                    if (lane == 0 && lo > i0) e0 = col_unstable(a, C, lo - 1, lo, nullptr, nullptr) ? 1 : 0;
                    if (lane == 1 && up < i1) e1 = col_unstable(a, C, up, up + 1, nullptr, nullptr) ? 1 : 0;
                    __syncwarp();
                    e0 = __shfl_sync(FULL_WARP, e0, 0);
                    e1 = __shfl_sync(FULL_WARP, e1, 1);
                    bool ext = false;
                    if (e0) { lo--; ext = true; }
                    if (e1) { up++; ext = true; }
                    if (!ext) break;
                }
                layers += up - lo + 1;
                changed = true;
                i = up;
            }
        }
        if (lane == 0 && passes >= 1 && (moist_t || dry_t)) {
            atomicAdd(&a.stats[2], (unsigned long long)moist_t);
            atomicAdd(&a.stats[3], (unsigned long long)dry_t);
        }
        if (fail) {
            if (lane == 0) atomicAdd(&a.stats[6], 1ull);
            __syncwarp();
            continue;
        }
        if (layers == 0) continue;
        if (a.relax < 1.0) {
            bool rok = true;
            for (int q = i0 + (int)lane; q <= i1; q += 32) {
                if (!C.touched[q] || !rok) continue;
                C.hL[q] = C.hL0[q] + a.relax * (C.hL[q] - C.hL0[q]);
                for (int g = 0; g < NG; g++) C.qt[q][g] = C.qt0[q][g] + a.relax * (C.qt[q][g] - C.qt0[q][g]);
                for (int r = 0; r < NT; r++) C.qr[q][r] = C.qr0[q][r] + a.relax * (C.qr[q][r] - C.qr0[q][r]);
                if (!col_settle(a, C, q)) rok = false;
            }
            rok = __all_sync(FULL_WARP, rok) != 0;
            __syncwarp();
            if (!rok) {
                if (lane == 0) atomicAdd(&a.stats[6], 1ull);
                __syncwarp();
                continue;
            }
        }
        for (int q = i0 + (int)lane; q <= i1; q += 32) {
            if (!C.touched[q]) continue;
            const size_t c = c0 + (size_t)q * plane;
            a.t[c] = C.T[q] / a.t_ref;
            for (int g = 0; g < NG; g++) {
                a.vap[g][c] = C.qv[q][g] * C.rho[q];
                a.cld[g][c] = C.qc[q][g] * C.rho[q];
                a.ice[g][c] = C.qi[q][g] * C.rho[q];
            }
            for (int r = 0; r < NT; r++) a.trf[r][c] = C.qr[q][r] * C.rho[q];
        }
        if (lane == 0) {
            atomicAdd(&a.stats[0], 1ull);
            atomicAdd(&a.stats[1], (unsigned long long)layers);
            atomicMax(&a.stats[7], (unsigned long long)passes);
        }
        __syncwarp();
    }
}

}  // namespace

int mca_setup(AtjupCtx* c) {
    const AtjupParams& P = c->P;
    if (P.im > MAXI) {
        set_error("set_mca: more than 64 radial levels are not supported");
        return ATJUP_ERR_UNSUPPORTED;
    }
    const size_t ncol = (size_t)P.jm * P.km;
    if (!c->mca_bounds) ATJUP_CUDA(cudaMalloc(&c->mca_bounds, sizeof(int2) * ncol));
    if (!c->mca_flags) ATJUP_CUDA(cudaMalloc(&c->mca_flags, sizeof(unsigned) * (2 * ncol + 1)));
    if (!c->mca_slots) ATJUP_CUDA(cudaMalloc(&c->mca_slots, sizeof(Col) * NSLOT));
    if (!c->mca_pairs) ATJUP_CUDA(cudaMalloc(&c->mca_pairs, (size_t)P.im * P.jm * P.km));
    if (!c->mca_stats) ATJUP_CUDA(cudaMalloc(&c->mca_stats, sizeof(unsigned long long) * (8 + 2 * NPART)));
    mca_bounds_kernel<<<dim3((P.km + 127) / 128, P.jm), 128, 0, c->stream>>>(
        c->solid, static_cast<int2*>(c->mca_bounds), P.im, P.jm, P.km, c->KP, c->mca.interior);
    c->launches++;
    ATJUP_CHECK_LAUNCH("mca_bounds");
    return ATJUP_OK;
}

int launch_mca(AtjupCtx* c) {
    const AtjupParams& P = c->P;
    const AtjupMca& M = c->mca;
    McaArgs a{};
    a.t = c->f[ATJUP_F_T];
    a.p_stat = c->f[ATJUP_F_P_STAT];
    a.rho_mix = c->f[ATJUP_F_RHO_MIX];
    a.vap[0] = c->f[ATJUP_F_H2O]; a.cld[0] = c->f[ATJUP_F_H2O_CLOUD]; a.ice[0] = c->f[ATJUP_F_H2O_ICE];
    a.vap[1] = c->f[ATJUP_F_NH3]; a.cld[1] = c->f[ATJUP_F_NH3_CLOUD]; a.ice[1] = c->f[ATJUP_F_NH3_ICE];
    a.trf[0] = c->f[ATJUP_F_H2S];
    a.trf[1] = c->f[ATJUP_F_NH4SH];
    a.solid = c->solid;
    a.layer_h = c->layer_h;
    a.bounds = static_cast<const int2*>(c->mca_bounds);
    a.gas[0] = c->micro.gas[0];
    a.gas[1] = c->micro.gas[1];
    a.tr_ep[0] = M.ep_h2s; a.tr_cond[0] = 0; a.tr_L[0] = 0.0;
    a.tr_ep[1] = 0.0;      a.tr_cond[1] = 1; a.tr_L[1] = M.L_nh4sh;
    a.cp = P.cp_mix;
    a.grav = P.g;
    a.t_ref = P.t_ref;
    a.r_mix = P.r_mix;
    a.relax = M.relax < 0.0 ? 0.0 : (M.relax > 1.0 ? 1.0 : M.relax);
    a.im = P.im; a.jm = P.jm; a.km = P.km; a.KP = c->KP;
    a.local_rho = P.local_rho;
    a.ledoux = M.ledoux;
    a.loading = M.loading;
    a.max_pass = M.max_pass > 0 ? M.max_pass : 64;
    const size_t ncol = (size_t)P.jm * P.km;
    a.stats = static_cast<unsigned long long*>(c->mca_stats);
    a.colflag = static_cast<unsigned*>(c->mca_flags);
    a.list = a.colflag + ncol;
    a.count = a.colflag + 2 * ncol;
    a.pairs = static_cast<uint8_t*>(c->mca_pairs);
    ATJUP_CUDA(cudaMemsetAsync(c->mca_stats, 0, sizeof(unsigned long long) * (8 + 2 * NPART), c->stream));
    ATJUP_CUDA(cudaMemsetAsync(a.colflag, 0, sizeof(unsigned) * ncol, c->stream));
    ATJUP_CUDA(cudaMemsetAsync(a.count, 0, sizeof(unsigned), c->stream));
    mca_census_kernel<<<dim3((P.km + 127) / 128, P.jm, P.im - 1), 128, 0, c->stream>>>(a);
    c->launches++;
    ATJUP_CHECK_LAUNCH("mca_census");
    // the listed columns (almost always none: the kernel then reads the count and returns; the
    // host does not wait for the count, so the launches of the step stay queued ahead)
    // (the two forms read the count and the one that does not apply returns at once)
    mca_column_warp_kernel<<<NSLOT / COL_WARPS, 32 * COL_WARPS, 0, c->stream>>>(a, static_cast<Col*>(c->mca_slots));
    c->launches++;
    ATJUP_CHECK_LAUNCH("mca_column_warp");
    mca_column_kernel<<<NSLOT / COL_BLOCK, COL_BLOCK, 0, c->stream>>>(a, static_cast<Col*>(c->mca_slots));
    c->launches++;
    ATJUP_CHECK_LAUNCH("mca_column");
    return ATJUP_OK;
}

// the counters of the last adjustment: [8], the census partials summed into [4] and [5]
int mca_read_stats(AtjupCtx* c, unsigned long long* out) {
    unsigned long long h[8 + 2 * NPART];
    ATJUP_CUDA(cudaMemcpyAsync(h, c->mca_stats, sizeof h, cudaMemcpyDeviceToHost, c->stream));
    ATJUP_CUDA(cudaStreamSynchronize(c->stream));
    for (int q = 0; q < 8; q++) out[q] = h[q];
    for (int q = 0; q < NPART; q++) { out[4] += h[8 + 2 * q]; out[5] += h[9 + 2 * q]; }
    return ATJUP_OK;
}

}  // namespace atjup
