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
// B200 form. Lexicographic SOR is replayed exactly as a pipelined wavefront: cell (a, b) of the
// box lies on the anti-diagonal d = a + b, its sweep-t update needs sweep t of (a-1, b) and
// (a, b-1) and sweep t-1 of (a+1, b) and (a, b+1), so step tau of the wavefront can update
// diagonal d = tau - 2(t-1) for every sweep t in flight at once. The cells of one step are then
// exactly the cells of one colour of the checkerboard, (a + b) = tau mod 2, less those whose sweep
// has not begun or is past the last; a step reads only the other colour, so the cells of a step
// are independent and one barrier between steps orders them. phi is stored split by colour (each
// row's cells of one colour contiguous), so a warp's lanes take consecutive cells of one row and
// read the four neighbours from consecutive words of the other colour.
//
// Each level is one thread-block cluster of C blocks (C = 4, or fewer when the GPU cannot hold
// every level's cluster at once: 26 levels on 104 SMs for the 41 x 181 x 361 grid). Block r owns
// a band of the box's rows with its phi, cell flags and per-cell constants in shared memory; the
// rows next to its band are read from the neighbouring blocks' shared memory (distributed shared
// memory), and a cluster barrier ends each step. Each sweep's largest change and largest |phi|
// are kept per block in a ring slot (the band's first cell of the sweep opens it, the other cells
// raise it by a shared-memory atomic maximum on the IEEE bit pattern, issued only when a cell
// exceeds the value it reads); sweep t is complete after step D + 2(t-1) (D = NJ + NK - 2), where
// every block reads the C slots and takes the stopping test. The sweeps after the converged one
// have by then already updated the first diagonals; each block restores its band from the newest
// snapshot that precedes them (one every SNAP_EVERY steps, in HBM) and the cluster replays up to
// the converged sweep. The arithmetic is the reference's, operation for operation (this file is
// compiled without FMA contraction), so the result is the reference's to the bit.
#include <algorithm>
#include <climits>
#include <cmath>
#include <vector>

#include <cooperative_groups.h>

#include "ctx.cuh"

namespace cg = cooperative_groups;

namespace atjup {

namespace {

constexpr double CONE_OMEGA = 1.9;       // InitValues_Jup.cpp:1726
constexpr int CONE_MAXIT = 40000;        // InitValues_Jup.cpp:1728
constexpr double CONE_TOL = 1.0e-10;     // InitValues_Jup.cpp:1761
constexpr int SNAP_EVERY = 64;           // wavefront steps between snapshots
constexpr int CONE_THREADS = 1024;
constexpr int CONE_CLUSTER = 4;          // blocks per level (fewer when the GPU cannot hold them)
constexpr size_t CONE_SMEM_CAP = 200 * 1024;
constexpr int NROW = 6;                  // per box row: aN, aS, aL, s, s dphi, A of a plain cell

// cell flags of the box (uint32 per cell: these bits, the special-cell index above bit 6)
enum : uint32_t { CF_SOLID = 1, CF_N = 2, CF_S = 4, CF_W = 8, CF_E = 16, CF_NEAR = 32 };
constexpr uint32_t CF_WALL = CF_N | CF_S | CF_W | CF_E;

}  // namespace

// One level's box. Colour-split storage: cell (a', b') of the box with its halo (a' = a + 1 in
// 0..NJ+1, b' = b + 1 in 0..NK+1) sits at ((c (NJ + 2) + a') PW + b' / 2), c = (a' + b') mod 2;
// the flags of interior cell (a, b) at ((c NJ + a) PW + (b + 1) / 2).
struct ConeLevel {
    int i, jlo, klo, NJ, NK, PW, D, n_spec;
    int64_t info_off;   // uint32 [2 * NJ * PW]: flags | special index << 6
    int64_t spec_off;   // int32 [n_spec]: (c NJ + a) PW + m of each special cell
    int64_t phi_off;    // double [2 * (NJ + 2) * PW] per warm-start buffer (halo included)
    int64_t snap_off;   // double [n_snap * C * 2 * (nbmax + 2) * PW]: per block, its band
    int64_t tab_off;    // double [2 * n_spec] (global-memory mode)
    int64_t row_off;    // double [NROW * NJ] (global-memory mode)
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
    int C = 1;                              // blocks (one cluster) per level
    int ring_max = 1;                       // the largest ring of the levels
    bool smem_mode = true;
    size_t smem = 0;                        // dynamic shared memory per block
    int64_t n_phi = 0;
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
    int jm, km, KP, H, smem_mode, C, ring_max;
    double dr, dthe, dphi;
};

// A block's band of a level's box as the kernel sees it. Local row la = 1..nb is box row
// a = A0 + la - 1 (halo coordinate a' = A0 + la); the words of colour x, local row la start at
// phi + x cs + la PW, la = 0 and nb + 1 being the rows beside the band (nrow, srow per colour:
// the neighbouring block's rows in its shared memory, or the box's halo).
struct Box {
    double* phi;
    int cs;                     // colour stride of phi
    const double* nrow[2];
    const double* srow[2];
    const uint32_t* info;       // flags of local row la, colour x at info + x ics + (la - 1) PW
    int ics;
    const double* tab;
    const double* rows;         // [NROW][NJ], indexed by box row
    unsigned long long* ring;   // [2 R]: largest change, largest |phi| of sweep t at t mod R
    int NJ, NK, PW, D, R;       // R a power of two
    int lgCH;                   // the row's words of one colour in 2^lgCH chunks of 32
    int nb, A0;
    bool div;
    double dthe, dphi;
};

__device__ __forceinline__ const double* row_of(const Box& B, int x, int la) {
    if (la == 0) return B.nrow[x];
    if (la == B.nb + 1) return B.srow[x];
    return B.phi + x * B.cs + la * B.PW;
}

// phi of the cell at local row la (0..nb+1), halo column b' (0..NK+1)
__device__ __forceinline__ double phi_at(const Box& B, int la, int bp) {
    return row_of(B, (B.A0 + la + bp) & 1, la)[bp >> 1];
}

// One SOR update of the cell at local row la, colour c, word m (InitValues_Jup.cpp:1739-1758), in
// the reference's order of operations. Returns false for a cell the sweep skips (solid, or no
// fluid face: A = 0); else the change and |phi| in dch, pabs.
__device__ __forceinline__ bool cone_update(const Box& B, int la, int c, int m, int off,
                                            double& dch, double& pabs) {
    const uint32_t inf = B.info[c * B.ics + (la - 1) * B.PW + m];
    if (inf & CF_SOLID) return false;
    const int a = B.A0 + la - 1;
    const double* rc = B.phi + (c ^ 1) * B.cs + la * B.PW;   // this row, the other colour
    const double pN = row_of(B, c ^ 1, la - 1)[m], pS = row_of(B, c ^ 1, la + 1)[m];
    const double pW = rc[m - 1 + off], pE = rc[m + off];
    const double aN = B.rows[a], aS = B.rows[B.NJ + a], aL = B.rows[2 * B.NJ + a];
    double A, Bs = 0.0;
    if (!(inf & (CF_WALL | CF_NEAR)) || (!B.div && !(inf & CF_WALL))) {
        // a plain cell: all four faces fluid
        A = B.rows[5 * B.NJ + a];
        Bs += aN * pN;
        Bs += aS * pS;
        Bs += aL * pW;
        Bs += aL * pE;
    } else if (B.div && (inf & CF_NEAR)) {
        A = 0.0;
        if (!(inf & CF_N)) { A += aN; Bs += aN * pN; }
        if (!(inf & CF_S)) { A += aS; Bs += aS * pS; }
        if (!(inf & CF_W)) { A += aL; Bs += aL * pW; }
        if (!(inf & CF_E)) { A += aL; Bs += aL * pE; }
        Bs += B.tab[2 * (inf >> 6)];
    } else {
        A = 0.0;
        const double vp = B.tab[2 * (inf >> 6)], wp = B.tab[2 * (inf >> 6) + 1];
        const double sj = B.rows[3 * B.NJ + a];
        if (inf & CF_N) Bs -= aN * B.dthe * (-vp); else { A += aN; Bs += aN * pN; }
        if (inf & CF_S) Bs -= aS * B.dthe * (vp);  else { A += aS; Bs += aS * pS; }
        if (inf & CF_W) Bs -= aL * sj * B.dphi * (-wp); else { A += aL; Bs += aL * pW; }
        if (inf & CF_E) Bs -= aL * sj * B.dphi * (wp);  else { A += aL; Bs += aL * pE; }
    }
    if (!(A > 0.0)) return false;
    double* own = B.phi + c * B.cs + la * B.PW + m;
    const double p = *own;
    const double pn = p + CONE_OMEGA * (Bs / A - p);
    dch = fabs(pn - p);
    *own = pn;
    pabs = fabs(pn);
    return true;
}

// std::max(cur, x) as the reference folds it (a NaN x leaves cur), on the ring's bit patterns
__device__ __forceinline__ void ring_raise(unsigned long long* slot, double x) {
    if (x > __longlong_as_double((long long)*(volatile unsigned long long*)slot))
        atomicMax(slot, (unsigned long long)__double_as_longlong(x));
}

// One cell of a wavefront step tau on the block's band: the cell of colour tau mod 2 at local row
// la, word m, if its sweep t = (tau - a - b) / 2 + 1 lies in [1, t_stop].
__device__ __forceinline__ void cone_cell(const Box& B, int tau, int t_stop, bool reduce, int la,
                                          int m) {
    const int c = tau & 1;
    const int a = B.A0 + la - 1;
    const int off = (c ^ (a + 1)) & 1;              // b' of word 0 of this colour in row a'
    const int b = off + 2 * m - 1;
    if (b < 0 || b >= B.NK) return;
    const int diff = tau - a - b;
    if (diff < 0) return;
    const int t = (diff >> 1) + 1;
    if (t > t_stop) return;
    double dch = 0.0, pabs = 0.0;
    const bool upd = cone_update(B, la, c, m, off, dch, pabs);
    if (!reduce) return;
    unsigned long long* slot = B.ring + 2 * (t & (B.R - 1));
    if (la == 1 && b == 0) {
        // the band's first cell of the sweep, alone in its sweep here at this step: opens the
        // band's slot
        slot[0] = (unsigned long long)__double_as_longlong(upd && dch > 0.0 ? dch : 0.0);
        slot[1] = (unsigned long long)__double_as_longlong(upd && pabs > 0.0 ? pabs : 0.0);
    } else if (upd) {
        ring_raise(slot, dch);
        ring_raise(slot + 1, pabs);
    }
}

// One wavefront step tau on the block's band. Warp w owns chunk w mod 2^lgCH of the local rows
// 1 + w / 2^lgCH + n 32 / 2^lgCH: lane l updates word 32 chunk + l of each (no division).
__device__ void cone_step(const Box& B, int tau, int t_stop, bool reduce) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m = ((warp & ((1 << B.lgCH) - 1)) << 5) + lane;
    const int la_step = (blockDim.x >> 5) >> B.lgCH;
    for (int la = 1 + (warp >> B.lgCH); la <= B.nb; la += la_step) cone_cell(B, tau, t_stop, reduce, la, m);
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

// the band's rows 1..nb of both colours between phi (colour stride cs) and a packed copy
// [2][nb][PW] (to_packed) or back
__device__ void band_copy(double* phi, int cs, double* packed, int nb, int PW, bool to_packed) {
    const int n = 2 * nb * PW;
    for (int x = threadIdx.x; x < n; x += blockDim.x) {
        const int col = x / (nb * PW), r = x - col * nb * PW;
        double* p = phi + col * cs + PW + r;      // local row 1 + r / PW, word r mod PW
        if (to_packed) packed[x] = *p;
        else *p = packed[x];
    }
}

// Lexicographic SOR of one level's solve as the pipelined wavefront on the cluster; returns the
// reference's sweep count `it` (the converged sweep, or CONE_MAXIT + 1 without convergence).
// snap: this block's snapshot ring, n_snap slots of 2 nbmax PW doubles. A cluster barrier ends
// every step: the next step's edge rows read the neighbours' rows of this one.
__device__ int cone_sor(const Box& B, double* snap, int slot_sz, int n_snap, int* snap_tag, int C) {
    cg::cluster_group cl = cg::this_cluster();
    band_copy(B.phi, B.cs, snap, B.nb, B.PW, true);
    if (threadIdx.x == 0) {
        snap_tag[0] = -1;
        for (int s = 1; s < n_snap; s++) snap_tag[s] = INT_MIN;
    }
    cl.sync();
    int next = 1 % n_snap, t_conv = 0, it = CONE_MAXIT + 1;
    for (int tau = 0;; tau++) {
        cone_step(B, tau, CONE_MAXIT, true);
        cl.sync();
        if (tau >= B.D && ((tau - B.D) & 1) == 0) {
            const int t = (tau - B.D) / 2 + 1;       // the sweep this step completed
            double dmax = 0.0, pmax = 0.0;
            for (int r = 0; r < C; r++) {
                const unsigned long long* sl = cl.map_shared_rank(B.ring + 2 * (t & (B.R - 1)), r);
                dmax = fmax(dmax, __longlong_as_double((long long)sl[0]));
                pmax = fmax(pmax, __longlong_as_double((long long)sl[1]));
            }
            if (dmax <= CONE_TOL * fmax(pmax, 1.0e-30)) { t_conv = t; break; }
            if (t == CONE_MAXIT) break;
        }
        if (tau % SNAP_EVERY == SNAP_EVERY - 1) {
            band_copy(B.phi, B.cs, snap + (size_t)next * slot_sz, B.nb, B.PW, true);
            if (threadIdx.x == 0) snap_tag[next] = tau;
            next = (next + 1) % n_snap;
            __syncthreads();
        }
    }
    if (t_conv > 0) {
        // back to the newest snapshot in which no cell is past sweep t_conv (the same slot in
        // every block), then replay with the sweeps capped at t_conv up to the step that
        // completes it
        it = t_conv;
        const int target = 2 * (t_conv - 1), tau_c = B.D + 2 * (t_conv - 1);
        int best = 0, btag = INT_MIN;
        for (int s = 0; s < n_snap; s++)
            if (snap_tag[s] != INT_MIN && snap_tag[s] <= target && snap_tag[s] > btag) { best = s; btag = snap_tag[s]; }
        band_copy(B.phi, B.cs, snap + (size_t)best * slot_sz, B.nb, B.PW, false);
        cl.sync();
        for (int tau = btag + 1; tau <= tau_c; tau++) {
            cone_step(B, tau, t_conv, false);
            cl.sync();
        }
    }
    return it;
}

__global__ void __launch_bounds__(CONE_THREADS, 1) cone_kernel(ConeArgs A) {
    extern __shared__ __align__(16) unsigned char cone_smem[];
    __shared__ int snap_tag[64];
    cg::cluster_group cl = cg::this_cluster();
    const int C = A.C;
    const int r = (int)cl.block_rank();
    const int lvl = blockIdx.x / C;
    const ConeLevel L = A.lv[lvl];
    const int NJ = L.NJ, NK = L.NK, PW = L.PW, i = L.i;
    const int A0 = (r * NJ) / C, nb = ((r + 1) * NJ) / C - A0, nbmax = (NJ + C - 1) / C;
    Box B;
    B.NJ = NJ; B.NK = NK; B.PW = PW; B.D = L.D; B.R = L.ring;
    B.nb = nb; B.A0 = A0;
    B.dthe = A.dthe; B.dphi = A.dphi;
    B.lgCH = 0;
    while ((32 << B.lgCH) < PW) B.lgCH++;
    B.ring = reinterpret_cast<unsigned long long*>(cone_smem);
    double* phi_local = reinterpret_cast<double*>(B.ring + 2 * A.ring_max);
    double *rows, *tab;
    if (A.smem_mode) {
        B.cs = (nbmax + 2) * PW;
        rows = phi_local + 2 * B.cs;
        tab = rows + NROW * NJ;
        uint32_t* inf = reinterpret_cast<uint32_t*>(tab + 2 * L.n_spec);
        B.ics = nbmax * PW;
        for (int x = threadIdx.x; x < 2 * nb * PW; x += blockDim.x) {
            const int col = x / (nb * PW), rr = x - col * nb * PW;
            inf[col * B.ics + rr] = A.info[L.info_off + (size_t)col * NJ * PW + (size_t)A0 * PW + rr];
        }
        B.info = inf;
        for (int x = 0; x < 2; x++) {
            B.nrow[x] = r > 0 ? cl.map_shared_rank(phi_local + x * B.cs + (A0 - ((r - 1) * NJ) / C) * PW, r - 1)
                              : phi_local + x * B.cs;
            B.srow[x] = r < C - 1 ? cl.map_shared_rank(phi_local + x * B.cs + PW, r + 1)
                                  : phi_local + x * B.cs + (nb + 1) * PW;
        }
    } else {
        // one block per level: phi in place in the warm-start buffer, the rest in HBM
        B.cs = (NJ + 2) * PW;
        rows = A.rows + L.row_off;
        tab = A.tab + L.tab_off;
        B.ics = NJ * PW;
        B.info = A.info + L.info_off;
    }
    B.tab = tab;
    B.rows = rows;
    // the row coefficients (InitValues_Jup.cpp:1733-1735) and A of a cell with four fluid faces
    for (int a = threadIdx.x; a < NJ; a += blockDim.x) {
        const int j = L.jlo + a;
        const double sj = A.s[j];
        const double aN = 0.5 * (sj + A.s[j - 1]) / (A.dthe * A.dthe);
        const double aS = 0.5 * (sj + A.s[j + 1]) / (A.dthe * A.dthe);
        const double aL = 1.0 / (sj * A.dphi * A.dphi);
        double a4 = 0.0;
        a4 += aN;
        a4 += aS;
        a4 += aL;
        a4 += aL;
        rows[a] = aN;
        rows[NJ + a] = aS;
        rows[2 * NJ + a] = aL;
        rows[3 * NJ + a] = sj;
        rows[4 * NJ + a] = sj * A.dphi;
        rows[5 * NJ + a] = a4;
    }
    const int32_t* spec = A.spec + L.spec_off;
    const int slot_sz = 2 * nbmax * PW;
    double* snap = A.snap + L.snap_off + (size_t)r * L.n_snap * slot_sz;
    if (A.H == 0 && r == 0 && threadIdx.x == 0) A.stats[2 * lvl] = 0;
    for (int pass = A.H > 0 ? 0 : 1; pass < 2; pass++) {
        B.div = pass == 0;
        double* prev = (B.div ? A.prev0 : A.prev1) + L.phi_off;
        if (A.smem_mode) {
            B.phi = phi_local;
            for (int x = threadIdx.x; x < 2 * PW; x += blockDim.x) {   // the rows beside the band
                const int col = x / PW, mm = x - col * PW;
                phi_local[col * B.cs + mm] = 0.0;
                phi_local[col * B.cs + (nb + 1) * PW + mm] = 0.0;
            }
            for (int x = threadIdx.x; x < 2 * nb * PW; x += blockDim.x) {
                const int col = x / (nb * PW), rr = x - col * nb * PW;
                phi_local[col * B.cs + PW + rr] = prev[(size_t)col * (NJ + 2) * PW + (size_t)(A0 + 1) * PW + rr];
            }
        } else {
            B.phi = prev + (size_t)A0 * PW;
            for (int x = 0; x < 2; x++) {
                B.nrow[x] = B.phi + x * B.cs;
                B.srow[x] = B.phi + x * B.cs + (nb + 1) * PW;
            }
        }
        // the per-cell constants of the band: the source of the divergence solve from the flow
        // before it, the wall-face velocities of the wall-flux solve from the flow it starts from
        __syncthreads();
        for (int x = threadIdx.x; x < L.n_spec; x += blockDim.x) {
            const int e = spec[x], mm = e % PW, rw = e / PW, a = rw % NJ, cc = rw / NJ;
            if (a < A0 || a >= A0 + nb) continue;
            const int b = ((cc ^ (a + 1)) & 1) + 2 * mm - 1;
            const int j = L.jlo + a, k = L.klo + b;
            if (B.div) {
                tab[2 * x] = (A.info[L.info_off + e] & CF_NEAR) ? cone_face_div(A, i, j, k) : 0.0;
            } else {
                const size_t cix = ((size_t)i * A.jm + j) * A.KP + k;
                tab[2 * x] = A.v[cix];
                tab[2 * x + 1] = A.w[cix];
            }
        }
        const int it = cone_sor(B, snap, slot_sz, L.n_snap, snap_tag, C);
        // v and w of the band incremented by the average of the two face corrections
        // (InitValues_Jup.cpp:1785-1793), a wall face's correction being minus the cell's velocity
        for (int x = threadIdx.x; x < nb * NK; x += blockDim.x) {
            const int la = 1 + x / NK, b = x - (la - 1) * NK;
            const int a = A0 + la - 1, bp = b + 1;
            const uint32_t inf = B.info[((a + b) & 1) * B.ics + (la - 1) * PW + (bp >> 1)];
            if (inf & CF_SOLID) continue;
            const size_t cix = ((size_t)i * A.jm + (L.jlo + a)) * A.KP + (L.klo + b);
            const double vp = A.v[cix], wp = A.w[cix], pp = phi_at(B, la, bp);
            const double sd = rows[4 * NJ + a];
            const double dN = (inf & CF_N) ? -vp : (pp - phi_at(B, la - 1, bp)) / A.dthe;
            const double dS = (inf & CF_S) ? -vp : (phi_at(B, la + 1, bp) - pp) / A.dthe;
            const double dW = (inf & CF_W) ? -wp : (pp - phi_at(B, la, bp - 1)) / sd;
            const double dE = (inf & CF_E) ? -wp : (phi_at(B, la, bp + 1) - pp) / sd;
            A.v[cix] = vp + 0.5 * (dN + dS);
            A.w[cix] = wp + 0.5 * (dW + dE);
        }
        // the band's phi is the warm start of the next call
        if (A.smem_mode)
            for (int x = threadIdx.x; x < 2 * nb * PW; x += blockDim.x) {
                const int col = x / (nb * PW), rr = x - col * nb * PW;
                prev[(size_t)col * (NJ + 2) * PW + (size_t)(A0 + 1) * PW + rr] = phi_local[col * B.cs + PW + rr];
            }
        if (r == 0 && threadIdx.x == 0) A.stats[2 * lvl + pass] = it;
        // the neighbours have read this band's edge rows before the next pass overwrites them
        cl.sync();
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
        L.PW = (L.NK + 3) / 2;                       // words per row and colour, halo included
        L.D = L.NJ + L.NK - 2;
        L.ring = 1;
        while (L.ring < L.D / 2 + 2) L.ring <<= 1;     // a power of two above the sweeps in flight
        L.n_snap = (L.D + SNAP_EVERY) / SNAP_EVERY + 2;
        if (L.n_snap > 64 || L.PW > 32 * 32) {
            delete cs;
            set_error("cone projection: box too large");
            return ATJUP_ERR_UNSUPPORTED;
        }
        L.info_off = (int64_t)info.size();
        L.spec_off = (int64_t)spec.size();
        info.resize(info.size() + 2 * (size_t)L.NJ * L.PW, CF_SOLID);   // unused words: skipped
        for (int a = 0; a < L.NJ; a++)
            for (int b = 0; b < L.NK; b++) {
                const int j = jlo + a, k = klo + b;
                const int e = (((a + b) & 1) * L.NJ + a) * L.PW + ((b + 1) >> 1);
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
                        spec.push_back(e);
                    }
                }
                info[L.info_off + e] = f;
            }
        L.n_spec = (int)(spec.size() - L.spec_off);
        const int64_t nphi = 2 * (int64_t)(L.NJ + 2) * L.PW;
        L.phi_off = n_phi;  n_phi += nphi;
        L.tab_off = n_tab;  n_tab += 2 * (int64_t)L.n_spec;
        L.row_off = n_row;  n_row += NROW * (int64_t)L.NJ;
        cs->ring_max = std::max(cs->ring_max, L.ring);
        cs->lv.push_back(L);
    }
    c->cone = cs;
    cs->n_phi = n_phi;
    const size_t nl = cs->lv.size();
    // blocks per level: a cluster of up to CONE_CLUSTER, each block a band of at least one row,
    // the bands in shared memory; a level whose box does not fit runs as one block in HBM
    int C = CONE_CLUSTER;
    for (const ConeLevel& L : cs->lv) C = std::min(C, L.NJ);
    auto smem_for = [&](int Cn) {
        size_t mx = 0;
        for (const ConeLevel& L : cs->lv) {
            const size_t nbmax = (size_t)(L.NJ + Cn - 1) / Cn;
            mx = std::max(mx, sizeof(double) * (2 * (nbmax + 2) * L.PW + NROW * (size_t)L.NJ +
                                                2 * (size_t)L.n_spec) +
                                  sizeof(uint32_t) * 2 * nbmax * L.PW);
        }
        return mx + sizeof(unsigned long long) * 2 * (size_t)cs->ring_max;
    };
    cs->smem_mode = nl > 0 && smem_for(std::max(C, 1)) <= CONE_SMEM_CAP;
    if (!cs->smem_mode) C = 1;
    C = std::max(C, 1);
    // the largest cluster for which the GPU holds every level's cluster at once
    for (; nl > 0 && C > 1; C--) {
        const size_t sm = smem_for(C);
        if (sm > CONE_SMEM_CAP) continue;
        if (cudaFuncSetAttribute(cone_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        cudaLaunchConfig_t cfg{};
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = C; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3((unsigned)(nl * C));
        cfg.blockDim = dim3(CONE_THREADS);
        cfg.dynamicSmemBytes = sm;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int n_active = 0;
        if (cudaOccupancyMaxActiveClusters(&n_active, cone_kernel, &cfg) == cudaSuccess &&
            n_active >= (int)nl)
            break;
        cudaGetLastError();
    }
    cs->smem = cs->smem_mode ? smem_for(C) : sizeof(unsigned long long) * 2 * (size_t)cs->ring_max;
    if (nl > 0)
        ATJUP_CUDA(cudaFuncSetAttribute(cone_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cs->smem));
    cs->C = C;
    for (ConeLevel& L : cs->lv) {
        const int64_t nbmax = (L.NJ + C - 1) / C;
        L.snap_off = n_snap;
        n_snap += (int64_t)C * L.n_snap * 2 * nbmax * L.PW;
    }
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
    if (!cs->smem_mode) {
        ATJUP_CUDA(cudaMalloc(&cs->tab, sizeof(double) * std::max<int64_t>(n_tab, 1)));
        ATJUP_CUDA(cudaMalloc(&cs->rows, sizeof(double) * n_row));
    }
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
        A.smem_mode = cs->smem_mode;
        A.C = cs->C;
        A.ring_max = cs->ring_max;
        A.dr = P.dr; A.dthe = P.dthe; A.dphi = P.dphi;
        cudaLaunchConfig_t cfg{};
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = cs->C; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3((unsigned)(cs->lv.size() * cs->C));
        cfg.blockDim = dim3(CONE_THREADS);
        cfg.dynamicSmemBytes = cs->smem;
        cfg.stream = c->stream;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        c->launches++;
        ATJUP_CUDA(cudaLaunchKernelEx(&cfg, cone_kernel, A));
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
