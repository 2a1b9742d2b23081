// fhd_batch.cu -- many independent 2D periodic boxes of uneven size solved
// together: one launch per multigrid level and operation covers every box.
//
// The reference solves one problem per process; a batch of independent
// realizations (the batched-realization workload: hundreds of 2D boxes of
// 32^2 .. 256^2) would otherwise be hundreds of contexts whose small levels
// leave the GPU idle between launches.  Here
//   * every array of a multigrid level is packed over the boxes that have
//     that level; a table of (box, tile) entries drives each per-level
//     launch, one CTA per 64x8 tile;
//   * the coarse end of each box's V-cycle runs in one CTA per box, in one
//     launch for all boxes (the single-CTA coarse kernels of fhd_coarse.cuh);
//   * GMRES runs per box with its scalar control (Arnoldi coefficients,
//     Givens rotations, stopping tests) on the device, one thread per box.
//     All boxes step through the same schedule -- the outer step, then the
//     inner slots 1..m -- and a box whose inner loop has stopped sits out
//     the remaining slots (masked), so its arithmetic is exactly what it
//     would do alone;
//   * dot products are per box: each tile stores its partial sum, and one
//     warp per box adds its tiles' partials in a fixed order, so a box's
//     result does not depend on the other boxes in the batch.
//
// Operators: dim 2, visc_type 1 with a constant viscosity eta per box,
// density 1 (alpha = 1, alphainv = 1), precon_type 1 (apply_precon.f90:
// 103-195 and the null-space step 429-460), one V-cycle per multigrid call.
// T is the multigrid precision (float in the mixed mode); the Krylov
// vectors and apply_matrix are FP64.
#include <algorithm>
#include <unordered_map>
#include <cmath>
#include <cstring>
#include <vector>

#include "fhd_solver.cuh"
#include "fhd_coarse.cuh"
#include "fhd_vec.cuh"

namespace fhd {
namespace bat {

constexpr int TX = 64, TY = 8;  // tile of a level: 64 x 8 cells, 32 x 8 threads
constexpr int MAXM = 16;        // gmres_max_inner
constexpr int MAXL = CS_MAXL;   // levels per box

struct Tile {
    int box, i0, j0;
};

// one box at one level: its grid and its offset in the level's packed arrays
struct Lev {
    Grid g;
    i64 off;
};

// which boxes an operation covers
enum Mode { M_ALL = 0, M_LIVE = 1, M_INNER = 2, M_PEND = 3, M_ZERO = 4 };

// GMRES state of one box (gmres.f90:32-619)
struct Ctl {
    int done, inner, pend, i, iter, total_iter, status, zero_x;
    double norm_b, norm_pre_b, norm_init_resid, norm_resid, norm_resid_Stokes, norm_init_Stokes, norm_resid_est;
    double abs_tol;
    double nrm[2];        // reduction results of the outer step
    double h[MAXM + 2];   // MGS results of the current inner slot: h[1..i], h[i+1] = |w|^2
    double H[(MAXM + 2) * (MAXM + 2)], cs[MAXM + 2], sn[MAXM + 2], s[MAXM + 2], y[MAXM + 2];
    double mean[3];       // null-space sums of the preconditioner
    double eta;           // the box's viscosity
    int i_exit, iters_acc;
};

__device__ __forceinline__ bool covers(const Ctl& c, int mode) {
    return mode == M_ALL     ? true
           : mode == M_LIVE  ? !c.done
           : mode == M_INNER ? c.inner != 0
           : mode == M_PEND  ? c.pend != 0
                             : c.zero_x != 0;
}

// Every tile kernel runs on a grid sized to the GPU (a few CTAs per SM), not
// one CTA per tile: a CTA owns the tiles q = blockIdx.x + r * gridDim.x of
// the launch's table.  In rounds of 256 each thread tests one of them
// against the mode, the covered ones are compacted in shared memory (in q
// order), and the whole CTA runs f(tile, q) on each in turn.  A box that
// sits out the operation then costs one load per tile instead of a CTA
// launch, and a covered tile's work is the CTA's 256 threads on its 64 x 8
// cells.  f is called by every thread of the CTA (it may synchronise); its
// return ends that thread's part of the tile.
template <class F>
__device__ __forceinline__ void for_tiles(const Tile* tiles, int n, const Ctl* ctl, int mode, F f) {
    __shared__ int s_q[256];
    __shared__ int s_w[8];
    const int tid = threadIdx.x + 32 * threadIdx.y;
    const int lane = tid & 31, w = tid >> 5;
    for (long long r0 = 0; (long long)blockIdx.x + r0 * gridDim.x < n; r0 += 256) {
        const long long q = (long long)blockIdx.x + (r0 + tid) * gridDim.x;
        bool live = false;
        if (q < n) live = mode == M_ALL || covers(ctl[tiles[q].box], mode);
        const unsigned bal = __ballot_sync(0xffffffffu, live);
        if (lane == 0) s_w[w] = __popc(bal);
        __syncthreads();
        int base = 0, tot = 0;
#pragma unroll
        for (int k = 0; k < 8; k++) {
            base += k < w ? s_w[k] : 0;
            tot += s_w[k];
        }
        if (live) s_q[base + __popc(bal & ((1u << lane) - 1u))] = (int)q;
        __syncthreads();
        for (int k = 0; k < tot; k++) {
            const int qq = s_q[k];
            f(tiles[qq], qq);
        }
        __syncthreads();
    }
}

// the staggered operator of a box at a level: alpha = 1 (a read-only array
// of ones), theta from the caller, the box's constant viscosity
template <typename T>
__device__ __forceinline__ StagOp<T> box_op(const T* ones, T theta, double eta, double dx) {
    StagOp<T> A;
    for (int c = 0; c < 3; c++) {
        A.alpha[c] = ones;
        A.bed[c] = ones;
    }
    A.alpha_scale = theta;
    A.beta = ones;
    A.gamma = ones;
    A.q = T(1.0 / (dx * dx));
    A.beta0_set = 1;
    A.beta0 = (T)eta;
    return A;
}

template <typename T>
__device__ __forceinline__ CCOp<T> box_ccop(const T* ones, double dx) {
    CCOp<T> A;
    for (int c = 0; c < 3; c++) A.a[c] = ones;
    A.q = T(1.0 / (dx * dx));
    return A;
}

// ---------------------------------------------------------------------
// staggered multigrid, per-level launches over (box, tile) tables
// ---------------------------------------------------------------------
// one colour of the 4-colour Gauss-Seidel (k_stag_gs): component C, faces
// with (i+j) % 2 == par
template <typename T, int C>
__global__ void __launch_bounds__(256) kb_stag_gs(const Tile* tiles, int n, const Lev* lev, int l, const Ctl* ctl, int mode,
                                                  T* const* phi, const T* const* rhs, const T* ones, T theta,
                                                  int par, T omega) {
    for_tiles(tiles, n, ctl, mode, [&](const Tile& t, int q) {
        const Lev L = lev[t.box * MAXL + l];
        const int j = t.j0 + threadIdx.y;
        const int i = t.i0 + 2 * threadIdx.x + ((j + par) & 1);
        if (j >= L.g.n[1] || i >= L.g.n[0]) return;
        CellF P;
        P.set(L.g, i, j, 0);
        T* p0 = phi[0] + L.off;
        T* p1 = phi[1] + L.off;
        const T* ph[3] = {p0, p1, nullptr};
        T* pc = C == 0 ? p0 : p1;
        const StagOp<T> A = box_op<T>(ones, theta, ctl[t.box].eta, L.g.dx);
        const i64 f = P.id(0, 0, 0);
        T dg;
        const T Lv = stag_lface<T, 2, 1, C>(A, ph, P, dg);
        pc[f] = pc[f] + sm_quot(omega * (ld(rhs[C] + L.off, f) - Lv), dg);
    });
}

// residual rhs - (theta alpha - L) phi of both components into tmp
template <typename T>
__global__ void __launch_bounds__(256) kb_stag_resid(const Tile* tiles, int n, const Lev* lev, int l, const Ctl* ctl,
                                                     int mode, T* const* phi, const T* const* rhs, T* const* tmp,
                                                     const T* ones, T theta) {
    for_tiles(tiles, n, ctl, mode, [&](const Tile& t, int q) {
        const Lev L = lev[t.box * MAXL + l];
        const int j = t.j0 + threadIdx.y;
        if (j >= L.g.n[1]) return;
        const StagOp<T> A = box_op<T>(ones, theta, ctl[t.box].eta, L.g.dx);
        const T* ph[3] = {phi[0] + L.off, phi[1] + L.off, nullptr};
    #pragma unroll
        for (int u = 0; u < 2; u++) {
            const int i = t.i0 + threadIdx.x + 32 * u;
            if (i >= L.g.n[0]) continue;
            CellF P;
            P.set(L.g, i, j, 0);
            const i64 f = P.id(0, 0, 0);
    #pragma unroll
            for (int c = 0; c < 2; c++) {
                T dg;
                const T Lv = stag_lface_c<T, 2, 1>(c, A, ph, P, dg);
                tmp[c][L.off + f] = ld(rhs[c] + L.off, f) - Lv;
            }
        }
    });
}

// stag_restriction of tmp (level l) into rhs (level l+1); the tiles are
// level l+1's
template <typename T>
__global__ void __launch_bounds__(256) kb_stag_restrict(const Tile* tiles, int n, const Lev* lev, int l, const Ctl* ctl,
                                                        int mode, T* const* tmp, T* const* crhs) {
    for_tiles(tiles, n, ctl, mode, [&](const Tile& t, int q) {
        const Lev F = lev[t.box * MAXL + l], Q = lev[t.box * MAXL + l + 1];
        const int j = t.j0 + threadIdx.y;
        if (j >= Q.g.n[1]) return;
    #pragma unroll
        for (int u = 0; u < 2; u++) {
            const int i = t.i0 + threadIdx.x + 32 * u;
            if (i >= Q.g.n[0]) continue;
            Cell X;
            X.nx = F.g.n[0]; X.ny = F.g.n[1]; X.nz = 1;
            X.i = 2 * i; X.j = 2 * j; X.k = 0;
            const i64 qc = (i64)i + (i64)Q.g.n[0] * j;
    #pragma unroll
            for (int c = 0; c < 2; c++) {
                const T* Fp = tmp[c] + F.off;
                crhs[c][Q.off + qc] = stag_restrict_expr<T, 2>(
                    0, [&](int o, int pa, int pb) { return ld(Fp, comp_off_id<2>(X, c, o, pa, pb)); });
            }
        }
    });
}

// stag_prolongation: fine phi (level l) += P coarse phi (level l+1); thread
// per fine face, the tiles are level l's; phi is the per-level table from
// level l on (phi[c] level l, phi[2 + c] level l+1)
template <typename T>
__global__ void __launch_bounds__(256) kb_stag_prolong(const Tile* tiles, int n, const Lev* lev, int l, const Ctl* ctl,
                                                       int mode, T* const* phi) {
    for_tiles(tiles, n, ctl, mode, [&](const Tile& t, int q) {
        const Lev F = lev[t.box * MAXL + l], Q = lev[t.box * MAXL + l + 1];
        const int j = t.j0 + threadIdx.y;
        if (j >= F.g.n[1]) return;
    #pragma unroll
        for (int u = 0; u < 2; u++) {
            const int i = t.i0 + threadIdx.x + 32 * u;
            if (i >= F.g.n[0]) continue;
            const int I[2] = {i, j};
            Cell H;
            H.nx = Q.g.n[0]; H.ny = Q.g.n[1]; H.nz = 1;
            H.i = i >> 1; H.j = j >> 1; H.k = 0;
            const i64 f = (i64)i + (i64)F.g.n[0] * j;
    #pragma unroll
            for (int c = 0; c < 2; c++) {
                const T* Cp = phi[2 + c] + Q.off;
                const int ca = (c == 0) ? 1 : 0;
                const int oa = (I[ca] & 1) ? 1 : -1;
                const T v = stag_prolong_expr<T, 2>((I[c] & 1) == 0, oa, 0, [&](int o, int pa, int pb) {
                    return ld(Cp, comp_off_id<2>(H, c, o, pa, pb));
                });
                T* Fp = phi[c] + F.off;
                Fp[f] = Fp[f] + v;
            }
        }
    });
}

// the coarse end of every covered box's V-cycle, one CTA per box
template <typename T>
__global__ void __launch_bounds__(CS_THREADS) kb_stag_coarse(const StagCoarseArgs<T>* args, const int* order,
                                                            const Ctl* ctl, int mode) {
    const int b = order[blockIdx.x];
    if (!covers(ctl[b], mode)) return;
    stag_coarse_run<T, 2, 1>(args[b]);
}

// ---------------------------------------------------------------------
// pressure multigrid
// ---------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) kb_cc_gsrb(const Tile* tiles, int n, const Lev* lev, int l, const Ctl* ctl, int mode,
                                                  T* phi, const T* rhs, const T* ones, int par) {
    for_tiles(tiles, n, ctl, mode, [&](const Tile& t, int q) {
        const Lev L = lev[t.box * MAXL + l];
        const int j = t.j0 + threadIdx.y;
        const int i = t.i0 + 2 * threadIdx.x + ((j + par) & 1);
        if (j >= L.g.n[1] || i >= L.g.n[0]) return;
        CellF P;
        P.set(L.g, i, j, 0);
        const CCOp<T> A = box_ccop<T>(ones, L.g.dx);
        T* ph = phi + L.off;
        T dg;
        const T Lv = cc_lap<T, 2>(A, ph, P, dg);
        const i64 f = P.id(0, 0, 0);
        ph[f] = ph[f] + sm_quot(ld(rhs + L.off, f) - Lv, dg);
    });
}

// residual of level l averaged onto level l+1's rhs; tiles of level l+1
template <typename T>
__global__ void __launch_bounds__(256) kb_cc_resid_restrict(const Tile* tiles, int n, const Lev* lev, int l, const Ctl* ctl,
                                                            int mode, const T* phi, const T* rhs, T* crhs,
                                                            const T* ones) {
    for_tiles(tiles, n, ctl, mode, [&](const Tile& t, int q) {
        const Lev F = lev[t.box * MAXL + l], Q = lev[t.box * MAXL + l + 1];
        const int j = t.j0 + threadIdx.y;
        if (j >= Q.g.n[1]) return;
        const CCOp<T> A = box_ccop<T>(ones, F.g.dx);
        const T* ph = phi + F.off;
        const T* rh = rhs + F.off;
    #pragma unroll
        for (int u = 0; u < 2; u++) {
            const int i = t.i0 + threadIdx.x + 32 * u;
            if (i >= Q.g.n[0]) continue;
            crhs[Q.off + (i64)i + (i64)Q.g.n[0] * j] = cc_resid_avg<T, 2>(
                A, F.g, i, j, 0, [&](i64 k) { return ld(ph, k); }, [&](i64 k) { return ld(rh, k); });
        }
    });
}

// phi (level l) += the parent cell's coarse phi (cphi, level l+1); tiles of
// level l
template <typename T>
__global__ void __launch_bounds__(256) kb_cc_prolong(const Tile* tiles, int n, const Lev* lev, int l, const Ctl* ctl,
                                                     int mode, T* phi, const T* cphi) {
    for_tiles(tiles, n, ctl, mode, [&](const Tile& t, int q) {
        const Lev F = lev[t.box * MAXL + l], Q = lev[t.box * MAXL + l + 1];
        const int j = t.j0 + threadIdx.y;
        if (j >= F.g.n[1]) return;
    #pragma unroll
        for (int u = 0; u < 2; u++) {
            const int i = t.i0 + threadIdx.x + 32 * u;
            if (i >= F.g.n[0]) continue;
            const T cv = ld(cphi + Q.off, (i64)(i >> 1) + (i64)Q.g.n[0] * (j >> 1));
            T* p = phi + F.off + (i64)i + (i64)F.g.n[0] * j;
            *p = *p + cv;
        }
    });
}

template <typename T>
__global__ void __launch_bounds__(CS_THREADS) kb_cc_coarse(const CCCoarseArgs<T>* args, const int* order,
                                                          const Ctl* ctl, int mode) {
    const int b = order[blockIdx.x];
    if (!covers(ctl[b], mode)) return;
    cc_coarse_run<T, 2>(args[b]);
}

// ---------------------------------------------------------------------
// preconditioner glue on level 0 (apply_precon.f90:103-195)
// ---------------------------------------------------------------------
// the multigrid rhs from the FP64 input: b_u in the precision of T
template <typename T>
__global__ void __launch_bounds__(256) kb_to_T(const Tile* tiles, int n, const Lev* lev, const Ctl* ctl, int mode,
                                               const double* const* b, T* const* out) {
    for_tiles(tiles, n, ctl, mode, [&](const Tile& t, int q) {
        const Lev L = lev[t.box * MAXL];
        const int j = t.j0 + threadIdx.y;
        if (j >= L.g.n[1]) return;
    #pragma unroll
        for (int u = 0; u < 2; u++) {
            const int i = t.i0 + threadIdx.x + 32 * u;
            if (i >= L.g.n[0]) continue;
            const i64 f = L.off + (i64)i + (i64)L.g.n[0] * j;
            out[0][f] = (T)b[0][f];
            out[1][f] = (T)b[1][f];
        }
    });
}

// mac_rhs = D x_u* + b_p (k_div_plus)
template <typename T>
__global__ void __launch_bounds__(256) kb_div_plus(const Tile* tiles, int n, const Lev* lev, const Ctl* ctl, int mode,
                                                   T* const* xu, const double* bp, T* out) {
    for_tiles(tiles, n, ctl, mode, [&](const Tile& t, int q) {
        const Lev L = lev[t.box * MAXL];
        const int j = t.j0 + threadIdx.y;
        if (j >= L.g.n[1]) return;
        const T dxinv = (T)(1.0 / L.g.dx);
        const T* u0 = xu[0] + L.off;
        const T* u1 = xu[1] + L.off;
    #pragma unroll
        for (int u = 0; u < 2; u++) {
            const int i = t.i0 + threadIdx.x + 32 * u;
            if (i >= L.g.n[0]) continue;
            CellF P;
            P.set(L.g, i, j, 0);
            const i64 f = P.id(0, 0, 0);
            const T s = (ld(u0, P.id(1, 0, 0)) - ld(u0, f)) * dxinv + (ld(u1, P.id(0, 1, 0)) - ld(u1, f)) * dxinv;
            out[L.off + f] = s + (T)bp[L.off + f];
        }
    });
}

// ---------------------------------------------------------------------
// per-box reductions: tile partials, then one warp per box in fixed order
// ---------------------------------------------------------------------
// sum over a 32 x 8 tile block in a fixed order (valid in thread (0, 0));
// every thread of the block calls it
__device__ __forceinline__ double tile_sum(double v) {
    __shared__ double sh[8];
    const int t = threadIdx.x + 32 * threadIdx.y;
    v = warp_sum(v);  // a warp is one row of the block
    if ((t & 31) == 0) sh[t >> 5] = v;
    __syncthreads();
    double s = 0.0;
    if (t == 0)
        for (int w = 0; w < 8; w++) s += sh[w];
    __syncthreads();  // sh is reused by the CTA's next tile
    return s;
}
// three sums at once, each in tile_sum's order (valid in thread (0, 0))
__device__ __forceinline__ void tile_sum3(double (&v)[3]) {
    __shared__ double sh3[3][8];
    const int t = threadIdx.x + 32 * threadIdx.y;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        v[c] = warp_sum(v[c]);
        if ((t & 31) == 0) sh3[c][t >> 5] = v[c];
    }
    __syncthreads();
    if (t == 0)
#pragma unroll
        for (int c = 0; c < 3; c++) {
            double s = 0.0;
            for (int w = 0; w < 8; w++) s += sh3[c][w];
            v[c] = s;
        }
    __syncthreads();  // sh3 is reused by the CTA's next tile
}

// x_u = x_u* - alphainv G Phi (k_sub_wgrad, alphainv = 1) and x_p = -beta
// mac_rhs + theta Phi (k_schur, kind 0, visc_type 1); with nsum > 0 also
// the tile sums of x_p, x_u, x_v (the first nsum of them) into part[c *
// pstride + tile], each added in the order of a separate sum pass over the
// stored values
template <typename T>
__global__ void __launch_bounds__(256) kb_precon_out(const Tile* tiles, int n, const Lev* lev, const Ctl* ctl, int mode,
                                                     T* const* xu, const T* Phi, const T* mac_rhs, double theta,
                                                     double* const* x, int nsum, double* part, i64 pstride) {
    for_tiles(tiles, n, ctl, mode, [&](const Tile& t, int q) {
        const Lev L = lev[t.box * MAXL];
        const int j = t.j0 + threadIdx.y;
        double sm[3] = {0.0, 0.0, 0.0};
        if (j < L.g.n[1]) {
            const T dxinv = (T)(1.0 / L.g.dx);
            const double eta = ctl[t.box].eta;
            const T* Ph = Phi + L.off;
    #pragma unroll
            for (int u = 0; u < 2; u++) {
                const int i = t.i0 + threadIdx.x + 32 * u;
                if (i >= L.g.n[0]) continue;
                CellF P;
                P.set(L.g, i, j, 0);
                const i64 f = P.id(0, 0, 0);
                const T pc = ld(Ph, f);
    #pragma unroll
                for (int c = 0; c < 2; c++) {
                    const T gp = (pc - ld(Ph, P.id(-(c == 0), -(c == 1), 0))) * dxinv;
                    const double xv = (double)(ld(xu[c] + L.off, f) + T(-1) * gp);
                    x[c][L.off + f] = xv;
                    sm[1 + c] += xv;
                }
                double v = (double)mac_rhs[L.off + f] * -1.0;
                v = v * eta;
                v = v + (double)pc * theta;
                x[2][L.off + f] = v;
                sm[0] += v;
            }
        }
        if (nsum > 0) {
            tile_sum3(sm);
            if (threadIdx.x == 0 && threadIdx.y == 0)
    #pragma unroll
                for (int c = 0; c < 3; c++)
                    if (c < nsum) part[c * pstride + q] = sm[c];
        }
    });
}

// sum over one box's tile partials into *dst(box)
template <class Dst>
__device__ __forceinline__ void seg_finish(const double* part, const int* t0, int box, Dst dst) {
    const int lane = threadIdx.x & 31;
    double s = 0.0;
    for (int q = t0[box] + lane; q < t0[box + 1]; q += 32) s += part[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) dst(s);
}

// one warp per box and field: ctl[b].<field which + c> = sum of its
// partials part[c * pstride + ..], c < ncomp
__global__ void __launch_bounds__(256) kb_seg_sum(int nbox, const double* part, i64 pstride, int ncomp, const int* t0,
                                                  Ctl* ctl, int mode, int which) {
    const int wg = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int box = wg / ncomp, comp = wg % ncomp;
    if (box >= nbox || !covers(ctl[box], mode)) return;
    const int fld = which + comp;
    seg_finish(part + comp * pstride, t0, box, [&](double s) {
        Ctl& c = ctl[box];
        if (fld < 2) c.nrm[fld] = s;
        else if (fld < 5) c.mean[fld - 2] = s;
        else c.h[fld - 5] = s;
    });
}

// weighted dot <a, b> (pressure weighted by wp2) of the 3 components, per tile
__global__ void __launch_bounds__(256) kb_dot(const Tile* tiles, int n, const Lev* lev, const Ctl* ctl, int mode,
                                              const double* const* a, const double* const* b, double wp2,
                                              double* part) {
    for_tiles(tiles, n, ctl, mode, [&](const Tile& t, int q) {
        const Lev L = lev[t.box * MAXL];
        const int j = t.j0 + threadIdx.y;
        double s = 0.0;
        if (j < L.g.n[1]) {
    #pragma unroll
            for (int u = 0; u < 2; u++) {
                const int i = t.i0 + threadIdx.x + 32 * u;
                if (i >= L.g.n[0]) continue;
                const i64 f = L.off + (i64)i + (i64)L.g.n[0] * j;
                double su = 0.0;
    #pragma unroll
                for (int c = 0; c < 3; c++) {
                    const double tt = a[c][f] * b[c][f];
                    su += c == 2 ? wp2 * tt : tt;
                }
                s += su;
            }
        }
        s = tile_sum(s);
        if (threadIdx.x == 0 && threadIdx.y == 0) part[q] = s;
    });
}

// x_p -= its box's mean (ctl.mean[0] / cells), and with ncomp = 3 also
// x_u, x_v (ctl.mean[1], mean[2])
__global__ void __launch_bounds__(256) kb_sub_means(const Tile* tiles, int n, const Lev* lev, const Ctl* ctl, int mode,
                                                    double* const* x, int ncomp) {
    for_tiles(tiles, n, ctl, mode, [&](const Tile& t, int q) {
        const Lev L = lev[t.box * MAXL];
        const int j = t.j0 + threadIdx.y;
        if (j >= L.g.n[1]) return;
        const Ctl& cb = ctl[t.box];
        const double cells = (double)L.g.nc;
        for (int c = 0; c < ncomp; c++) {
            const double m = cb.mean[c] / cells;
            double* a = x[c == 0 ? 2 : c - 1] + L.off + (i64)L.g.n[0] * j;
    #pragma unroll
            for (int u = 0; u < 2; u++) {
                const int i = t.i0 + threadIdx.x + 32 * u;
                if (i < L.g.n[0]) a[i] = a[i] - m;
            }
        }
    });
}

// ---------------------------------------------------------------------
// apply_matrix and the Krylov vector passes (FP64)
// ---------------------------------------------------------------------
// out = A x (mode 0) or rhs - A x (mode 1) (k_stokes_apply)
__global__ void __launch_bounds__(256) kb_stokes_apply(const Tile* tiles, int n, const Lev* lev, const Ctl* ctl, int mode,
                                                       const double* const* x, const double* const* rhs,
                                                       double* const* out, int amode, const double* ones,
                                                       double theta) {
    for_tiles(tiles, n, ctl, mode, [&](const Tile& t, int q) {
        const Lev L = lev[t.box * MAXL];
        const int j = t.j0 + threadIdx.y;
        if (j >= L.g.n[1]) return;
        const StagOp<double> A = box_op<double>(ones, theta, ctl[t.box].eta, L.g.dx);
        const double dxinv = 1.0 / L.g.dx;
        const double* phi[3] = {x[0] + L.off, x[1] + L.off, nullptr};
        const double* p = x[2] + L.off;
    #pragma unroll
        for (int u = 0; u < 2; u++) {
            const int i = t.i0 + threadIdx.x + 32 * u;
            if (i >= L.g.n[0]) continue;
            CellF P;
            P.set(L.g, i, j, 0);
            const i64 f = P.id(0, 0, 0);
            const double pc = ld(p, f);
            double div = 0.0;
    #pragma unroll
            for (int c = 0; c < 2; c++) {
                double dg;
                double Lv = stag_lface_c<double, 2, 1>(c, A, phi, P, dg);
                const double gp = (pc - ld(p, P.id(-(c == 0), -(c == 1), 0))) * dxinv;
                Lv = Lv + gp;
                out[c][L.off + f] = amode ? ld(rhs[c] + L.off, f) - Lv : Lv;
                div += (ld(phi[c], P.id(c == 0, c == 1, 0)) - ld(phi[c], f)) * dxinv;
            }
            const double bp = div * -1.0;
            out[2][L.off + f] = amode ? ld(rhs[2] + L.off, f) - bp : bp;
        }
    });
}

// Modified Gram-Schmidt pass k (k_mgs): w -= h[k-1] V_{k-2} (k > 1), then
// the tile's partial of <w, V_{k-1}> (or <w, w> when vnext is null)
__global__ void __launch_bounds__(256) kb_mgs(const Tile* tiles, int n, const Lev* lev, const Ctl* ctl, double* const* w,
                                              const double* const* vprev, int hk, const double* const* vnext,
                                              double wp2, double* part) {
    for_tiles(tiles, n, ctl, M_INNER, [&](const Tile& t, int q) {
        const Lev L = lev[t.box * MAXL];
        const double h = vprev ? ctl[t.box].h[hk] : 0.0;
        const int j = t.j0 + threadIdx.y;
        double s = 0.0;
        if (j < L.g.n[1]) {
    #pragma unroll
            for (int u = 0; u < 2; u++) {
                const int i = t.i0 + threadIdx.x + 32 * u;
                if (i >= L.g.n[0]) continue;
                const i64 f = L.off + (i64)i + (i64)L.g.n[0] * j;
                double su = 0.0;
    #pragma unroll
                for (int c = 0; c < 3; c++) {
                    double x = w[c][f];
                    if (vprev) {
                        x = x - vprev[c][f] * h;
                        w[c][f] = x;
                    }
                    const double y = vnext ? vnext[c][f] : x;
                    const double tt = x * y;
                    su += c == 2 ? wp2 * tt : tt;
                }
                s += su;
            }
        }
        s = tile_sum(s);
        if (threadIdx.x == 0 && threadIdx.y == 0) part[q] = s;
    });
}

// v = w / |w| with |w| = sqrt(ctl.h[hk]) (k_scale_by_norm), or w / norm_resid
// (k_scale_div, hk < 0)
__global__ void __launch_bounds__(256) kb_scale(const Tile* tiles, int n, const Lev* lev, const Ctl* ctl,
                                                double* const* v, const double* const* w, int hk) {
    for_tiles(tiles, n, ctl, M_INNER, [&](const Tile& t, int q) {
        const Ctl& c = ctl[t.box];
        const Lev L = lev[t.box * MAXL];
        const int j = t.j0 + threadIdx.y;
        if (j >= L.g.n[1]) return;
        const double d = hk < 0 ? c.norm_resid : sqrt(c.h[hk]);
    #pragma unroll
        for (int u = 0; u < 2; u++) {
            const int i = t.i0 + threadIdx.x + 32 * u;
            if (i >= L.g.n[0]) continue;
            const i64 f = L.off + (i64)i + (i64)L.g.n[0] * j;
    #pragma unroll
            for (int q = 0; q < 3; q++) v[q][f] = w[q][f] / d;
        }
    });
}

// x += sum_k y_k V_{k-1} over the box's exit index (k_update_sol)
__global__ void __launch_bounds__(256) kb_update_sol(const Tile* tiles, int n, const Lev* lev, const Ctl* ctl,
                                                     double* const* x, const double* V, i64 vstride, i64 cstride) {
    for_tiles(tiles, n, ctl, M_PEND, [&](const Tile& t, int q) {
        const Ctl& c = ctl[t.box];
        const Lev L = lev[t.box * MAXL];
        const int j = t.j0 + threadIdx.y;
        if (j >= L.g.n[1]) return;
        const int m = c.i_exit;
    #pragma unroll
        for (int u = 0; u < 2; u++) {
            const int i = t.i0 + threadIdx.x + 32 * u;
            if (i >= L.g.n[0]) continue;
            const i64 f = L.off + (i64)i + (i64)L.g.n[0] * j;
            double acc[3] = {x[0][f], x[1][f], x[2][f]};
            for (int it = 0; it < m; it++) {
                const double yi = c.y[it + 1];
    #pragma unroll
                for (int q = 0; q < 3; q++) acc[q] = acc[q] + V[it * vstride + (i64)q * cstride + f] * yi;
            }
    #pragma unroll
            for (int q = 0; q < 3; q++) x[q][f] = acc[q];
        }
    });
}

// x = 0 for the boxes whose rhs is below gmres_abs_tol (gmres.f90:166-172)
__global__ void __launch_bounds__(256) kb_zero_x(const Tile* tiles, int n, const Lev* lev, const Ctl* ctl,
                                                 double* const* x) {
    for_tiles(tiles, n, ctl, M_ZERO, [&](const Tile& t, int q) {
        const Lev L = lev[t.box * MAXL];
        const int j = t.j0 + threadIdx.y;
        if (j >= L.g.n[1]) return;
    #pragma unroll
        for (int u = 0; u < 2; u++) {
            const int i = t.i0 + threadIdx.x + 32 * u;
            if (i >= L.g.n[0]) continue;
            const i64 f = L.off + (i64)i + (i64)L.g.n[0] * j;
            x[0][f] = 0.0;
            x[1][f] = 0.0;
            x[2][f] = 0.0;
        }
    });
}

// ---------------------------------------------------------------------
// GMRES control, one thread per box (gmres.f90:137-491)
// ---------------------------------------------------------------------
struct GParams {
    double rel_tol, wp;
    int m, max_iter, min_iter, max_outer;
};

// one warp per box: the control block zeroed word by word, keeping the
// accumulated iteration count
__global__ void kb_ctl_reset(int nbox, Ctl* ctl, const double* eta, const double* abs_tol) {
    const int b = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (b >= nbox) return;
    Ctl& c = ctl[b];
    const int acc = c.iters_acc;
    __syncwarp();
    unsigned long long* w = reinterpret_cast<unsigned long long*>(&c);
    static_assert(sizeof(Ctl) % 8 == 0, "Ctl is a whole number of 8-byte words");
    for (int k = lane; k < (int)(sizeof(Ctl) / 8); k += 32) w[k] = 0ull;
    __syncwarp();
    if (lane == 0) {
        c.iters_acc = acc;
        c.eta = eta[b];
        c.abs_tol = abs_tol[b];
    }
}

// after |M^-1 b|^2 (nrm[0]) and |b|^2 (nrm[1])
__global__ void kb_ctl_init(int nbox, Ctl* ctl) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nbox) return;
    Ctl& c = ctl[b];
    c.norm_pre_b = sqrt(c.nrm[0]);
    c.norm_b = sqrt(c.nrm[1]);
    if (c.norm_b <= c.abs_tol) {
        c.done = 1;
        c.zero_x = 1;
    }
}

// the outer step's stopping tests, after |b - A x|^2 (nrm[0]) and
// |M^-1 (b - A x)|^2 (nrm[1])
__global__ void kb_ctl_outer(int nbox, Ctl* ctl, GParams P) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nbox) return;
    Ctl& c = ctl[b];
    if (c.done) return;
    c.norm_resid_Stokes = sqrt(c.nrm[0]);
    c.norm_resid = sqrt(c.nrm[1]);
    if (c.iter == 0) {
        c.norm_init_Stokes = c.norm_resid_Stokes;
        c.norm_init_resid = c.norm_resid;
        c.norm_resid_est = c.norm_resid;
    }
    bool stop = false;
    if (c.total_iter >= P.max_iter) {
        c.status = FHD_WARN_NOT_CONVERGED_MAXITER;
        stop = true;
    } else if (c.total_iter >= P.min_iter) {
        if (c.norm_resid <= P.rel_tol * fmin(c.norm_pre_b, c.norm_init_resid)) {
            if (c.norm_resid_Stokes >= 10 * P.rel_tol * fmin(c.norm_b, c.norm_init_Stokes))
                c.status = FHD_WARN_TRUE_RESID;
            stop = true;
        } else if (c.norm_resid <= c.abs_tol) {
            stop = true;
        }
    }
    if (!stop && c.iter >= P.max_outer) {
        c.status = FHD_WARN_NOT_CONVERGED_OUTER;
        stop = true;
    }
    if (stop) {
        c.done = 1;
        c.iters_acc += c.total_iter;
        return;
    }
    c.iter++;
    for (int k = 0; k < MAXM + 2; k++) c.s[k] = 0.0;
    c.s[1] = c.norm_resid;
    c.inner = 1;
    c.i = 0;
}

// after inner slot i's MGS: the Hessenberg column, Givens rotations and the
// residual estimate (least_squares, rotmat, gmres.f90:531-597); at the
// loop's end, SolveUTriangular (599-619) and the pending solution update
__global__ void kb_ctl_inner(int nbox, Ctl* ctl, int i, GParams P) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nbox) return;
    Ctl& c = ctl[b];
    if (!c.inner) return;
    const int W = MAXM + 2;
    auto Hh = [&](int r, int q) -> double& { return c.H[r * W + q]; };
    c.total_iter++;
    c.i = i;
    for (int k = 1; k <= i; k++) Hh(k, i) = c.h[k];
    Hh(i + 1, i) = sqrt(c.h[i + 1]);
    for (int k = 1; k <= i - 1; k++) {
        const double tt = c.cs[k] * Hh(k, i) + c.sn[k] * Hh(k + 1, i);
        Hh(k + 1, i) = -c.sn[k] * Hh(k, i) + c.cs[k] * Hh(k + 1, i);
        Hh(k, i) = tt;
    }
    {
        const double a = Hh(i, i), bb = Hh(i + 1, i);
        if (bb == 0.0) {
            c.cs[i] = 1.0;
            c.sn[i] = 0.0;
        } else if (fabs(bb) > fabs(a)) {
            const double tt = a / bb;
            c.sn[i] = 1.0 / sqrt(1.0 + tt * tt);
            c.cs[i] = tt * c.sn[i];
        } else {
            const double tt = bb / a;
            c.cs[i] = 1.0 / sqrt(1.0 + tt * tt);
            c.sn[i] = tt * c.cs[i];
        }
        const double tt = c.cs[i] * c.s[i];
        c.s[i + 1] = -c.sn[i] * c.s[i];
        c.s[i] = tt;
        Hh(i, i) = c.cs[i] * Hh(i, i) + c.sn[i] * Hh(i + 1, i);
        Hh(i + 1, i) = 0.0;
    }
    c.norm_resid_est = fabs(c.s[i + 1]);
    bool brk = i == P.m;
    if (c.total_iter >= P.max_iter) brk = true;
    else if (c.total_iter >= P.min_iter)
        if (c.norm_resid_est <= P.rel_tol * fmin(c.norm_pre_b, c.norm_init_resid) || c.norm_resid_est <= c.abs_tol)
            brk = true;
    if (!brk) return;
    const int k = i - 1;
    c.y[k + 1] = c.s[k + 1] / Hh(k + 1, k + 1);
    for (int ii = k; ii >= 1; ii--) {
        double acc = 0.0;
        for (int jj = ii + 1; jj <= k + 1; jj++) acc += Hh(ii, jj) * c.y[jj];
        c.y[ii] = (c.s[ii] - acc) / Hh(ii, ii);
    }
    c.i_exit = i;
    c.inner = 0;
    c.pend = 1;
}

__global__ void kb_ctl_clear_pend(int nbox, Ctl* ctl) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < nbox) ctl[b].pend = 0;
}

__global__ void kb_count_live(int nbox, const Ctl* ctl, int* live) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < nbox && !ctl[b].done) atomicAdd(live, 1);
}

// ---------------------------------------------------------------------
// the overdamped step's glue (advance_timestep_overdamped.f90:135-734,
// one species: density 1 throughout)
// ---------------------------------------------------------------------
// N(0,1) per element from Philox-4x32-10 keyed by (seed, box), counter
// (element, field, step): Box-Muller, the cosine branch
__device__ __forceinline__ uint32_t mulhi32(uint32_t a, uint32_t b) {
    return (uint32_t)(((uint64_t)a * (uint64_t)b) >> 32);
}
__device__ __forceinline__ void philox10(uint32_t (&c)[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        const uint32_t hi0 = mulhi32(0xD2511F53u, c[0]), lo0 = 0xD2511F53u * c[0];
        const uint32_t hi1 = mulhi32(0xCD9E8D57u, c[2]), lo1 = 0xCD9E8D57u * c[2];
        const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}
__device__ __forceinline__ double normal_at(uint64_t seed, int box, uint32_t e, uint32_t field, uint32_t step) {
    uint32_t c[4] = {e, field, step, (uint32_t)box};
    philox10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const uint64_t a = ((uint64_t)c[0] << 32) | c[1], bb = ((uint64_t)c[2] << 32) | c[3];
    const double u1 = (double)((a >> 11) + 1) * 0x1.0p-53;
    const double u2 = (double)(bb >> 11) * 0x1.0p-53;
    return sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
}

struct StepNoise {
    uint64_t seed;
    uint32_t step;
    double w[2];     // stage weights of the two random stages
    double var_fac;  // variance_coef_mom * 2 / (dV * h), times k_B T per box
};

// rhs_v = -G p + div(stochastic stress) + eta Lap u, rhs_p = div u
// (the overdamped stage's right-hand side); the random stress of stage r:
// cell entries sqrt(2) N(0,1) (field 2r + c), node entries N(0,1) (field
// 4 + r) shared by the two components, scaled by sqrt(var_fac kT eta)
template <typename T>
__global__ void __launch_bounds__(256) kb_step_rhs(const Tile* tiles, int n, const Lev* lev, const Ctl* ctl,
                                                   const double* const* u, const double* p, double* const* rv,
                                                   double* rp, const double* ones, const double* kT, StepNoise N) {
    for_tiles(tiles, n, ctl, M_ALL, [&](const Tile& t, int q) {
        const Lev L = lev[t.box * MAXL];
        const int j = t.j0 + threadIdx.y;
        if (j >= L.g.n[1]) return;
        const double eta = ctl[t.box].eta;
        const StagOp<double> A = box_op<double>(ones, 0.0, eta, L.g.dx);
        const double dxinv = 1.0 / L.g.dx;
        const double* phi[3] = {u[0] + L.off, u[1] + L.off, nullptr};
        const double* pp = p + L.off;
        const T amp = (T)(sqrt(N.var_fac * kT[t.box]) * sqrt(eta));
        const int nx = L.g.n[0], ny = L.g.n[1];
        auto cell_w = [&](int ci, int cj, int comp) -> T {
            const uint32_t e = (uint32_t)(wrapc(ci, nx) + nx * wrapc(cj, ny));
            T s = T(0);
            for (int r = 0; r < 2; r++)
                if (N.w[r] != 0.0)
                    s = s + (T)N.w[r] * (T)(1.4142135623730951 * normal_at(N.seed, t.box, e, 2 * r + comp, N.step));
            return amp * s;
        };
        auto node_w = [&](int ci, int cj) -> T {
            const uint32_t e = (uint32_t)(wrapc(ci, nx) + nx * wrapc(cj, ny));
            T s = T(0);
            for (int r = 0; r < 2; r++)
                if (N.w[r] != 0.0) s = s + (T)N.w[r] * (T)normal_at(N.seed, t.box, e, 4 + r, N.step);
            return amp * s;
        };
    #pragma unroll
        for (int uu = 0; uu < 2; uu++) {
            const int i = t.i0 + threadIdx.x + 32 * uu;
            if (i >= nx) continue;
            CellF P;
            P.set(L.g, i, j, 0);
            const i64 f = P.id(0, 0, 0);
            const T dxi = (T)dxinv;
            T dv[2];
            dv[0] = (cell_w(i, j, 0) - cell_w(i - 1, j, 0)) * dxi + (node_w(i, j + 1) - node_w(i, j)) * dxi;
            dv[1] = (node_w(i + 1, j) - node_w(i, j)) * dxi + (cell_w(i, j, 1) - cell_w(i, j - 1, 1)) * dxi;
            const double pc = ld(pp, f);
            double div = 0.0;
    #pragma unroll
            for (int c = 0; c < 2; c++) {
                double dg;
                const double Lu = stag_lface_c<double, 2, 1>(c, A, phi, P, dg);  // -eta Lap u
                const double gp = (pc - ld(pp, P.id(-(c == 0), -(c == 1), 0))) * dxinv;
                double v = -gp;
                v = v + (double)dv[c];
                v = v + Lu * -1.0;
                rv[c][L.off + f] = v;
                div += (ld(phi[c], P.id(c == 0, c == 1, 0)) - ld(phi[c], f)) * dxinv;
            }
            rp[L.off + f] = div;
        }
    });
}

// u += du, p += dp
__global__ void __launch_bounds__(256) kb_axpy3(const Tile* tiles, int n, const Lev* lev, double* const* a,
                                                const double* const* d) {
    for_tiles(tiles, n, nullptr, M_ALL, [&](const Tile& t, int q) {
        const Lev L = lev[t.box * MAXL];
        const int j = t.j0 + threadIdx.y;
        if (j >= L.g.n[1]) return;
    #pragma unroll
        for (int u = 0; u < 2; u++) {
            const int i = t.i0 + threadIdx.x + 32 * u;
            if (i >= L.g.n[0]) continue;
            const i64 f = L.off + (i64)i + (i64)L.g.n[0] * j;
    #pragma unroll
            for (int q = 0; q < 3; q++) a[q][f] = a[q][f] + d[q][f];
        }
    });
}

__global__ void kb_set_abs_tol(int nbox, const Ctl* ctl, double* abs_tol, double base, double rel) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < nbox) abs_tol[b] = fmax(base, ctl[b].norm_pre_b * rel);
}

}  // namespace bat
}  // namespace fhd

using namespace fhd;
using namespace fhd::bat;

// =====================================================================
// host side
// =====================================================================
struct fhd_batch {
    int nbox = 0;
    int prec = FHD_PREC_FP64;
    double dx = 1.0;
    fhd_gmres_params p;
    cudaStream_t stream = nullptr;
    int sms = 148, smem_optin = 232448;
    std::vector<int> nx, ny, nls, nlc, lcs, lcc;
    int Ls = 0, Lc = 0;                // most levels of any box
    std::vector<void*> allocs;         // every device allocation
    Lev* dlev_s = nullptr;             // [nbox * MAXL]
    Lev* dlev_c = nullptr;
    // per-level launch tables: boxes whose level l is above their coarse end
    std::vector<Tile*> tab_s, tab_c;
    std::vector<int> ntab_s, ntab_c;
    // restriction targets: level l of the boxes that reach it by launches
    // (l <= their coarse end), so that the coarse kernel's first level is
    // included
    std::vector<Tile*> all_s, all_c;
    std::vector<int> nall_s, nall_c;
    Tile* tab0 = nullptr;              // every box's level-0 tiles
    int ntab0 = 0;
    int* dt0 = nullptr;                // first level-0 tile of each box
    std::vector<i64> Ns, Nc;           // packed sizes per level
    // multigrid arrays (precision T), per level: stag phi/rhs/tmp x2; cc phi/rhs/tmp
    std::vector<void*> sphi, srhs, stmp;  // [l*2 + c]
    std::vector<void*> cphi, crhs, ctmp;  // [l]
    void** dsphi = nullptr;               // device pointer tables [l*2 + c]
    void** dsrhs = nullptr;
    void** dstmp = nullptr;
    void* ones = nullptr;                 // max level-0 cells of T ones
    double* ones64 = nullptr;
    void* sargs = nullptr;                // StagCoarseArgs<T>[nbox]
    void* cargs = nullptr;                // CCCoarseArgs<T>[nbox]
    std::vector<unsigned char> sargs_h;   // host copy of sargs
    size_t smem_s = 0, smem_c = 0;
    // coarse-kernel CTA -> box, the boxes with the largest coarse hierarchy
    // first (they set the launch's length; the small ones fill in behind)
    int* ord_s = nullptr;
    int* ord_c = nullptr;
    // FP64 level-0 vectors, three components each: b, x, r, w, tmp, V (m+1)
    i64 N0 = 0;
    double* vec = nullptr;                // all FP64 vectors
    double** dvp = nullptr;               // device pointer tables, 3 per vector
    int m = 5;
    Ctl* ctl = nullptr;
    double* part = nullptr;               // tile partials
    double* deta = nullptr;
    double* dabs = nullptr;
    int* dlive = nullptr;
    int* hlive = nullptr;                 // pinned
    // step work: du, rhs (FP64, three components each)
    double* step = nullptr;
    double* dkT = nullptr;
    long long launches = 0;
    std::unordered_map<const void*, int> occ;  // resident CTAs per SM of each tile kernel
    // GMRES launch sequences as CUDA graphs: init, outer, inner (see gmres)
    cudaGraphExec_t gx[3] = {nullptr, nullptr, nullptr};
    long long gn[3] = {0, 0, 0};  // kernels in each
    int g_ok = 0;
    double g_theta = 0.0;
};

namespace {

template <typename T>
T* dalloc(fhd_batch* B, i64 n) {
    void* p = nullptr;
    if (cudaMalloc(&p, sizeof(T) * (size_t)(n > 0 ? n : 1)) != cudaSuccess) return nullptr;
    B->allocs.push_back(p);
    return (T*)p;
}

int nlevs(int nx, int ny, int minwidth) {
    Grid g;
    g.dim = 2;
    g.n[0] = nx;
    g.n[1] = ny;
    g.n[2] = 1;
    g.nc = (i64)nx * ny;
    g.dx = 1.0;
    return nlevs_mg(g, minwidth);
}

Grid grid2(int nx, int ny, double dx) {
    Grid g;
    g.dim = 2;
    g.n[0] = nx;
    g.n[1] = ny;
    g.n[2] = 1;
    g.nc = (i64)nx * ny;
    g.dx = dx;
    return g;
}

void tiles_of(std::vector<Tile>& v, int box, int nx, int ny) {
    for (int j0 = 0; j0 < ny; j0 += TY)
        for (int i0 = 0; i0 < nx; i0 += TX) v.push_back(Tile{box, i0, j0});
}

template <typename T>
int build(fhd_batch* B) {
    const int nb = B->nbox;
    const size_t budget = (size_t)B->smem_optin;
    // levels of every box, their grids and packed offsets
    std::vector<Lev> ls((size_t)nb * MAXL), lc((size_t)nb * MAXL);
    B->Ls = B->Lc = 0;
    for (int b = 0; b < nb; b++) {
        B->Ls = std::max(B->Ls, B->nls[b]);
        B->Lc = std::max(B->Lc, B->nlc[b]);
    }
    B->Ns.assign(B->Ls, 0);
    B->Nc.assign(B->Lc, 0);
    for (int b = 0; b < nb; b++) {
        int nx = B->nx[b], ny = B->ny[b];
        double dx = B->dx;
        for (int l = 0; l < B->nls[b]; l++) {
            ls[(size_t)b * MAXL + l] = Lev{grid2(nx, ny, dx), B->Ns[l]};
            B->Ns[l] += (i64)nx * ny;
            nx /= 2;
            ny /= 2;
            dx *= 2.0;
        }
        nx = B->nx[b];
        ny = B->ny[b];
        dx = B->dx;
        for (int l = 0; l < B->nlc[b]; l++) {
            lc[(size_t)b * MAXL + l] = Lev{grid2(nx, ny, dx), B->Nc[l]};
            B->Nc[l] += (i64)nx * ny;
            nx /= 2;
            ny /= 2;
            dx *= 2.0;
        }
        // the coarse ends: the first level from which every coarser one fits
        // one CTA's shared memory (3 dim arrays per staggered level, 3 per
        // pressure level)
        auto first = [&](int nl, const std::vector<Lev>& v, int per) {
            size_t acc = 0;
            int f = nl;
            for (int l = nl - 1; l >= 0; l--) {
                acc += (size_t)per * (size_t)v[(size_t)b * MAXL + l].g.nc * sizeof(T);
                if (acc > budget || nl - l > CS_MAXL) break;
                f = l;
            }
            return f;
        };
        B->lcs[b] = first(B->nls[b], ls, 6);
        B->lcc[b] = first(B->nlc[b], lc, 3);
        // the bottom level is always inside the coarse kernel
        if (B->lcs[b] >= B->nls[b] || B->lcc[b] >= B->nlc[b]) return FHD_ERR_UNSUPPORTED;
        // levels above the coarse end are smoothed by colour launches, which
        // need even extents
        for (int l = 0; l < B->lcs[b]; l++) {
            const Grid& g = ls[(size_t)b * MAXL + l].g;
            if ((g.n[0] & 1) || (g.n[1] & 1)) return FHD_ERR_UNSUPPORTED;
        }
        for (int l = 0; l < B->lcc[b]; l++) {
            const Grid& g = lc[(size_t)b * MAXL + l].g;
            if ((g.n[0] & 1) || (g.n[1] & 1)) return FHD_ERR_UNSUPPORTED;
        }
    }
    B->N0 = B->Ns[0];
    // launch tables
    auto upload_tiles = [&](const std::vector<Tile>& v) -> Tile* {
        Tile* d = dalloc<Tile>(B, (i64)v.size());
        if (d && !v.empty()) cudaMemcpy(d, v.data(), sizeof(Tile) * v.size(), cudaMemcpyHostToDevice);
        return d;
    };
    B->tab_s.assign(B->Ls, nullptr);
    B->ntab_s.assign(B->Ls, 0);
    B->all_s.assign(B->Ls, nullptr);
    B->nall_s.assign(B->Ls, 0);
    for (int l = 0; l < B->Ls; l++) {
        std::vector<Tile> v, a;
        for (int b = 0; b < nb; b++) {
            if (l >= B->nls[b]) continue;
            const Grid& g = ls[(size_t)b * MAXL + l].g;
            if (l < B->lcs[b]) tiles_of(v, b, g.n[0], g.n[1]);
            if (l >= 1 && l <= B->lcs[b]) tiles_of(a, b, g.n[0], g.n[1]);
        }
        B->ntab_s[l] = (int)v.size();
        B->tab_s[l] = upload_tiles(v);
        B->nall_s[l] = (int)a.size();
        B->all_s[l] = upload_tiles(a);
    }
    B->tab_c.assign(B->Lc, nullptr);
    B->ntab_c.assign(B->Lc, 0);
    B->all_c.assign(B->Lc, nullptr);
    B->nall_c.assign(B->Lc, 0);
    for (int l = 0; l < B->Lc; l++) {
        std::vector<Tile> v, a;
        for (int b = 0; b < nb; b++) {
            if (l >= B->nlc[b]) continue;
            const Grid& g = lc[(size_t)b * MAXL + l].g;
            if (l < B->lcc[b]) tiles_of(v, b, g.n[0], g.n[1]);
            if (l >= 1 && l <= B->lcc[b]) tiles_of(a, b, g.n[0], g.n[1]);
        }
        B->ntab_c[l] = (int)v.size();
        B->tab_c[l] = upload_tiles(v);
        B->nall_c[l] = (int)a.size();
        B->all_c[l] = upload_tiles(a);
    }
    {
        std::vector<Tile> v;
        std::vector<int> t0(nb + 1, 0);
        for (int b = 0; b < nb; b++) {
            t0[b] = (int)v.size();
            tiles_of(v, b, B->nx[b], B->ny[b]);
        }
        t0[nb] = (int)v.size();
        B->ntab0 = (int)v.size();
        B->tab0 = upload_tiles(v);
        B->dt0 = dalloc<int>(B, nb + 1);
        if (!B->dt0) return FHD_ERR_OOM;
        cudaMemcpy(B->dt0, t0.data(), sizeof(int) * (nb + 1), cudaMemcpyHostToDevice);
    }
    B->dlev_s = dalloc<Lev>(B, (i64)nb * MAXL);
    B->dlev_c = dalloc<Lev>(B, (i64)nb * MAXL);
    if (!B->dlev_s || !B->dlev_c) return FHD_ERR_OOM;
    cudaMemcpy(B->dlev_s, ls.data(), sizeof(Lev) * ls.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(B->dlev_c, lc.data(), sizeof(Lev) * lc.size(), cudaMemcpyHostToDevice);
    // multigrid arrays
    B->sphi.assign(2 * B->Ls, nullptr);
    B->srhs.assign(2 * B->Ls, nullptr);
    B->stmp.assign(2 * B->Ls, nullptr);
    for (int l = 0; l < B->Ls; l++)
        for (int c = 0; c < 2; c++) {
            B->sphi[2 * l + c] = dalloc<T>(B, B->Ns[l]);
            B->srhs[2 * l + c] = dalloc<T>(B, B->Ns[l]);
            B->stmp[2 * l + c] = dalloc<T>(B, B->Ns[l]);
            if (!B->sphi[2 * l + c] || !B->srhs[2 * l + c] || !B->stmp[2 * l + c]) return FHD_ERR_OOM;
        }
    B->cphi.assign(B->Lc, nullptr);
    B->crhs.assign(B->Lc, nullptr);
    B->ctmp.assign(B->Lc, nullptr);
    for (int l = 0; l < B->Lc; l++) {
        B->cphi[l] = dalloc<T>(B, B->Nc[l]);
        B->crhs[l] = dalloc<T>(B, B->Nc[l]);
        B->ctmp[l] = dalloc<T>(B, B->Nc[l]);
        if (!B->cphi[l] || !B->crhs[l] || !B->ctmp[l]) return FHD_ERR_OOM;
    }
    B->dsphi = dalloc<void*>(B, 2 * B->Ls);
    B->dsrhs = dalloc<void*>(B, 2 * B->Ls);
    B->dstmp = dalloc<void*>(B, 2 * B->Ls);
    if (!B->dsphi || !B->dsrhs || !B->dstmp) return FHD_ERR_OOM;
    cudaMemcpy(B->dsphi, B->sphi.data(), sizeof(void*) * 2 * B->Ls, cudaMemcpyHostToDevice);
    cudaMemcpy(B->dsrhs, B->srhs.data(), sizeof(void*) * 2 * B->Ls, cudaMemcpyHostToDevice);
    cudaMemcpy(B->dstmp, B->stmp.data(), sizeof(void*) * 2 * B->Ls, cudaMemcpyHostToDevice);
    i64 nmax = 1;
    for (int b = 0; b < nb; b++) nmax = std::max(nmax, (i64)B->nx[b] * B->ny[b]);
    {
        std::vector<T> h((size_t)nmax, T(1));
        std::vector<double> h64((size_t)nmax, 1.0);
        B->ones = dalloc<T>(B, nmax);
        B->ones64 = dalloc<double>(B, nmax);
        if (!B->ones || !B->ones64) return FHD_ERR_OOM;
        cudaMemcpy(B->ones, h.data(), sizeof(T) * nmax, cudaMemcpyHostToDevice);
        cudaMemcpy(B->ones64, h64.data(), sizeof(double) * nmax, cudaMemcpyHostToDevice);
    }
    // coarse-kernel arguments per box
    std::vector<StagCoarseArgs<T>> sa(nb);
    std::vector<CCCoarseArgs<T>> ca(nb);
    B->smem_s = B->smem_c = 0;
    for (int b = 0; b < nb; b++) {
        StagCoarseArgs<T>& a = sa[b];
        memset(&a, 0, sizeof(a));
        const int l0 = B->lcs[b];
        a.nlev = B->nls[b] - l0;
        a.load_phi = l0 == 0;
        a.n_down = B->p.stag_mg_nsmooths_down;
        a.n_up = B->p.stag_mg_nsmooths_up;
        a.n_bottom = B->p.stag_mg_nsmooths_bottom;
        a.jacobi = B->p.stag_mg_smoother == 0;
        a.omega = (T)B->p.stag_mg_omega;
        for (int c = 0; c < 2; c++) {
            a.phi[c] = (T*)B->sphi[2 * l0 + c] + ls[(size_t)b * MAXL + l0].off;
            a.rhs[c] = (const T*)B->srhs[2 * l0 + c] + ls[(size_t)b * MAXL + l0].off;
        }
        size_t off = 0;
        for (int q = 0; q < a.nlev; q++) {
            const Grid& g = ls[(size_t)b * MAXL + l0 + q].g;
            a.g[q] = g;
            StagOp<T>& A = a.A[q];
            for (int c = 0; c < 3; c++) {
                A.alpha[c] = (const T*)B->ones;
                A.bed[c] = (const T*)B->ones;
            }
            A.alpha_scale = T(0);  // set per solve (theta)
            A.beta = (const T*)B->ones;
            A.gamma = (const T*)B->ones;
            A.q = T(1.0 / (g.dx * g.dx));
            A.beta0_set = 1;
            A.beta0 = T(1);  // set per solve (eta)
            a.off[q] = (int)off;
            off += (size_t)6 * (size_t)g.nc;
        }
        B->smem_s = std::max(B->smem_s, off * sizeof(T));
        CCCoarseArgs<T>& cq = ca[b];
        memset(&cq, 0, sizeof(cq));
        const int m0 = B->lcc[b];
        cq.nlev = B->nlc[b] - m0;
        cq.load_phi = m0 == 0;
        cq.n_down = B->p.mg_nsmooths_down;
        cq.n_up = B->p.mg_nsmooths_up;
        cq.n_bottom = B->p.mg_nsmooths_bottom;
        cq.phi = (T*)B->cphi[m0] + lc[(size_t)b * MAXL + m0].off;
        cq.rhs = (const T*)B->crhs[m0] + lc[(size_t)b * MAXL + m0].off;
        off = 0;
        for (int q = 0; q < cq.nlev; q++) {
            const Grid& g = lc[(size_t)b * MAXL + m0 + q].g;
            cq.g[q] = g;
            for (int c = 0; c < 3; c++) cq.A[q].a[c] = (const T*)B->ones;
            cq.A[q].q = T(1.0 / (g.dx * g.dx));
            cq.off[q] = (int)off;
            off += (size_t)3 * (size_t)g.nc;
        }
        B->smem_c = std::max(B->smem_c, off * sizeof(T));
    }
    B->sargs = dalloc<StagCoarseArgs<T>>(B, nb);
    B->cargs = dalloc<CCCoarseArgs<T>>(B, nb);
    if (!B->sargs || !B->cargs) return FHD_ERR_OOM;
    cudaMemcpy(B->sargs, sa.data(), sizeof(StagCoarseArgs<T>) * nb, cudaMemcpyHostToDevice);
    cudaMemcpy(B->cargs, ca.data(), sizeof(CCCoarseArgs<T>) * nb, cudaMemcpyHostToDevice);
    {
        std::vector<int> os(nb), oc(nb);
        for (int b = 0; b < nb; b++) os[b] = oc[b] = b;
        auto work = [&](const std::vector<Lev>& v, int b, int l0) { return v[(size_t)b * MAXL + l0].g.nc; };
        std::stable_sort(os.begin(), os.end(),
                         [&](int a, int b) { return work(ls, a, B->lcs[a]) > work(ls, b, B->lcs[b]); });
        std::stable_sort(oc.begin(), oc.end(),
                         [&](int a, int b) { return work(lc, a, B->lcc[a]) > work(lc, b, B->lcc[b]); });
        B->ord_s = dalloc<int>(B, nb);
        B->ord_c = dalloc<int>(B, nb);
        if (!B->ord_s || !B->ord_c) return FHD_ERR_OOM;
        cudaMemcpy(B->ord_s, os.data(), sizeof(int) * nb, cudaMemcpyHostToDevice);
        cudaMemcpy(B->ord_c, oc.data(), sizeof(int) * nb, cudaMemcpyHostToDevice);
    }
    B->sargs_h.resize(sizeof(StagCoarseArgs<T>) * nb);
    memcpy(B->sargs_h.data(), sa.data(), B->sargs_h.size());
    if (B->smem_s > budget || B->smem_c > budget) return FHD_ERR_UNSUPPORTED;
    if (cudaFuncSetAttribute(kb_stag_coarse<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)B->smem_s) !=
            cudaSuccess ||
        cudaFuncSetAttribute(kb_cc_coarse<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)B->smem_c) !=
            cudaSuccess)
        return FHD_ERR_CUDA;
    // FP64 vectors: b, x, r, w, tmp, du-rhs pair for the step, V (m+1)
    const int nvec = 5 + (B->m + 1);
    B->vec = dalloc<double>(B, (i64)nvec * 3 * B->N0);
    B->dvp = dalloc<double*>(B, (i64)nvec * 3);
    B->step = dalloc<double>(B, (i64)6 * B->N0);
    B->ctl = dalloc<Ctl>(B, nb);
    B->part = dalloc<double>(B, 3 * B->ntab0);  // three fields of tile partials
    B->deta = dalloc<double>(B, nb);
    B->dabs = dalloc<double>(B, nb);
    B->dkT = dalloc<double>(B, nb);
    B->dlive = dalloc<int>(B, 1);
    if (!B->vec || !B->dvp || !B->step || !B->ctl || !B->part || !B->deta || !B->dabs || !B->dkT || !B->dlive)
        return FHD_ERR_OOM;
    std::vector<double*> hp((size_t)nvec * 3);
    for (int v = 0; v < nvec; v++)
        for (int c = 0; c < 3; c++) hp[(size_t)v * 3 + c] = B->vec + ((i64)v * 3 + c) * B->N0;
    cudaMemcpy(B->dvp, hp.data(), sizeof(double*) * hp.size(), cudaMemcpyHostToDevice);
    cudaMemset(B->ctl, 0, sizeof(Ctl) * nb);
    if (cudaMallocHost((void**)&B->hlive, sizeof(int)) != cudaSuccess) return FHD_ERR_OOM;
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : FHD_ERR_CUDA;
}

// vector v (0 b, 1 x, 2 r, 3 w, 4 tmp, 5.. V_0..V_m) as a device pointer table
double* const* vp(fhd_batch* B, int v) { return B->dvp + (size_t)v * 3; }
double* vc(fhd_batch* B, int v, int c) { return B->vec + ((i64)v * 3 + c) * B->N0; }
enum { V_B = 0, V_X = 1, V_R = 2, V_W = 3, V_TMP = 4, V_V0 = 5 };

inline int post(fhd_batch* B) {
    B->launches++;
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) {
        set_last_error(std::string("batched kernel launch: ") + cudaGetErrorString(e));
        return FHD_ERR_CUDA;
    }
    return 0;
}
#define BPOST(B)                 \
    do {                         \
        int rc_ = post(B);       \
        if (rc_) return rc_;     \
    } while (0)

const dim3 TB(32, 8, 1);

// grid of a tile kernel (for_tiles): its resident CTAs on every SM, at most
// one CTA per tile
template <class K>
int tgrid(fhd_batch* B, K kern, int n) {
    const void* key = reinterpret_cast<const void*>(kern);
    auto it = B->occ.find(key);
    int per = 1;
    if (it == B->occ.end()) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, 256, 0) != cudaSuccess || per < 1) per = 1;
        B->occ[key] = per;
    } else {
        per = it->second;
    }
    return std::max(1, std::min(n, per * B->sms));
}

// per-box sum of the tile partials into ctl.<which>
int seg(fhd_batch* B, int mode, int which, int ncomp = 1) {
    kb_seg_sum<<<(B->nbox * ncomp * 32 + 255) / 256, 256, 0, B->stream>>>(B->nbox, B->part, (i64)B->ntab0, ncomp,
                                                                          B->dt0, B->ctl, mode, which);
    BPOST(B);
    return 0;
}

template <typename T>
int stag_smooth(fhd_batch* B, int l, int mode, T theta, int count) {
    if (!B->ntab_s[l]) return 0;
    T* const* phi = (T* const*)(B->dsphi + 2 * l);
    const T* const* rhs = (const T* const*)(B->dsrhs + 2 * l);
    const T omega = (T)B->p.stag_mg_omega;
    for (int s = 0; s < count; s++)
        for (int color = 1; color <= 4; color++) {
            const int par = (color + 1) & 1;
            if (color <= 2)
                kb_stag_gs<T, 0><<<tgrid(B, kb_stag_gs<T, 0>, B->ntab_s[l]), TB, 0, B->stream>>>(B->tab_s[l], B->ntab_s[l], B->dlev_s, l, B->ctl, mode, phi,
                                                                    rhs, (const T*)B->ones, theta, par, omega);
            else
                kb_stag_gs<T, 1><<<tgrid(B, kb_stag_gs<T, 1>, B->ntab_s[l]), TB, 0, B->stream>>>(B->tab_s[l], B->ntab_s[l], B->dlev_s, l, B->ctl, mode, phi,
                                                                    rhs, (const T*)B->ones, theta, par, omega);
            BPOST(B);
        }
    return 0;
}

// one staggered V-cycle of every covered box (stag_mg_solver.f90:323-808),
// level-0 phi and rhs in the packed level-0 arrays
template <typename T>
int stag_vcycle(fhd_batch* B, int mode, T theta) {
    cudaStream_t st = B->stream;
    for (int l = 1; l < B->Ls; l++)
        for (int c = 0; c < 2; c++)
            if (cudaMemsetAsync(B->sphi[2 * l + c], 0, sizeof(T) * B->Ns[l], st) != cudaSuccess) return FHD_ERR_CUDA;
    for (int l = 0; l + 1 < B->Ls; l++) {
        if (!B->ntab_s[l]) continue;
        int rc = stag_smooth<T>(B, l, mode, theta, B->p.stag_mg_nsmooths_down);
        if (rc) return rc;
        kb_stag_resid<T><<<tgrid(B, kb_stag_resid<T>, B->ntab_s[l]), TB, 0, st>>>(B->tab_s[l], B->ntab_s[l], B->dlev_s, l, B->ctl, mode,
                                                       (T* const*)(B->dsphi + 2 * l), (const T* const*)(B->dsrhs + 2 * l),
                                                       (T* const*)(B->dstmp + 2 * l), (const T*)B->ones, theta);
        BPOST(B);
        // the restriction's targets: level l+1 of the boxes smoothing level l
        // by launches (it may be their coarse kernel's first level)
        kb_stag_restrict<T><<<tgrid(B, kb_stag_restrict<T>, B->nall_s[l + 1]), TB, 0, st>>>(B->all_s[l + 1], B->nall_s[l + 1], B->dlev_s, l, B->ctl, mode,
                                                            (T* const*)(B->dstmp + 2 * l),
                                                            (T* const*)(B->dsrhs + 2 * (l + 1)));
        BPOST(B);
    }
    kb_stag_coarse<T><<<B->nbox, CS_THREADS, B->smem_s, st>>>((const StagCoarseArgs<T>*)B->sargs, B->ord_s, B->ctl,
                                                              mode);
    BPOST(B);
    for (int l = B->Ls - 2; l >= 0; l--) {
        if (!B->ntab_s[l]) continue;
        kb_stag_prolong<T><<<tgrid(B, kb_stag_prolong<T>, B->ntab_s[l]), TB, 0, st>>>(B->tab_s[l], B->ntab_s[l], B->dlev_s, l, B->ctl, mode,
                                                         (T* const*)(B->dsphi + 2 * l));
        BPOST(B);
        int rc = stag_smooth<T>(B, l, mode, theta, B->p.stag_mg_nsmooths_up);
        if (rc) return rc;
    }
    return 0;
}

// Phi = 0, one pressure V-cycle of every covered box on cc level 0's rhs
template <typename T>
int cc_vcycle(fhd_batch* B, int mode) {
    cudaStream_t st = B->stream;
    for (int l = 0; l < B->Lc; l++)
        if (cudaMemsetAsync(B->cphi[l], 0, sizeof(T) * B->Nc[l], st) != cudaSuccess) return FHD_ERR_CUDA;
    auto smooth = [&](int l, int count) -> int {
        for (int s = 0; s < count; s++)
            for (int par = 0; par < 2; par++) {
                kb_cc_gsrb<T><<<tgrid(B, kb_cc_gsrb<T>, B->ntab_c[l]), TB, 0, st>>>(B->tab_c[l], B->ntab_c[l], B->dlev_c, l, B->ctl, mode, (T*)B->cphi[l],
                                                          (const T*)B->crhs[l], (const T*)B->ones, par);
                BPOST(B);
            }
        return 0;
    };
    for (int l = 0; l + 1 < B->Lc; l++) {
        if (!B->ntab_c[l]) continue;
        int rc = smooth(l, B->p.mg_nsmooths_down);
        if (rc) return rc;
        kb_cc_resid_restrict<T><<<tgrid(B, kb_cc_resid_restrict<T>, B->nall_c[l + 1]), TB, 0, st>>>(B->all_c[l + 1], B->nall_c[l + 1], B->dlev_c, l, B->ctl, mode,
                                                                (const T*)B->cphi[l], (const T*)B->crhs[l],
                                                                (T*)B->crhs[l + 1], (const T*)B->ones);
        BPOST(B);
    }
    kb_cc_coarse<T><<<B->nbox, CS_THREADS, B->smem_c, st>>>((const CCCoarseArgs<T>*)B->cargs, B->ord_c, B->ctl,
                                                            mode);
    BPOST(B);
    for (int l = B->Lc - 2; l >= 0; l--) {
        if (!B->ntab_c[l]) continue;
        kb_cc_prolong<T><<<tgrid(B, kb_cc_prolong<T>, B->ntab_c[l]), TB, 0, st>>>(B->tab_c[l], B->ntab_c[l], B->dlev_c, l, B->ctl, mode, (T*)B->cphi[l],
                                                      (const T*)B->cphi[l + 1]);
        BPOST(B);
        int rc = smooth(l, B->p.mg_nsmooths_up);
        if (rc) return rc;
    }
    return 0;
}

// x = M^-1 b (precon_type 1) for the covered boxes; b, x: vector indices
template <typename T>
int precon(fhd_batch* B, int bv, int xv, int mode, double theta) {
    cudaStream_t st = B->stream;
    // level-0 velocity unknowns start at zero, rhs = b_u
    for (int c = 0; c < 2; c++)
        if (cudaMemsetAsync(B->sphi[c], 0, sizeof(T) * B->N0, st) != cudaSuccess) return FHD_ERR_CUDA;
    kb_to_T<T><<<tgrid(B, kb_to_T<T>, B->ntab0), TB, 0, st>>>(B->tab0, B->ntab0, B->dlev_s, B->ctl, mode, vp(B, bv), (T* const*)B->dsrhs);
    BPOST(B);
    int rc = stag_vcycle<T>(B, mode, (T)theta);
    if (rc) return rc;
    kb_div_plus<T><<<tgrid(B, kb_div_plus<T>, B->ntab0), TB, 0, st>>>(B->tab0, B->ntab0, B->dlev_s, B->ctl, mode, (T* const*)B->dsphi, vc(B, bv, 2),
                                            (T*)B->crhs[0]);
    BPOST(B);
    if ((rc = cc_vcycle<T>(B, mode))) return rc;
    // null space (apply_precon.f90:429-460): mean of p, and of u when theta
    // = 0, summed per tile by the output pass
    const int ncomp = theta == 0.0 ? 3 : 1;
    kb_precon_out<T><<<tgrid(B, kb_precon_out<T>, B->ntab0), TB, 0, st>>>(
        B->tab0, B->ntab0, B->dlev_s, B->ctl, mode, (T* const*)B->dsphi, (const T*)B->cphi[0], (const T*)B->crhs[0],
        theta, vp(B, xv), ncomp, B->part, (i64)B->ntab0);
    BPOST(B);
    if ((rc = seg(B, mode, 2, ncomp))) return rc;
    kb_sub_means<<<tgrid(B, kb_sub_means, B->ntab0), TB, 0, st>>>(B->tab0, B->ntab0, B->dlev_s, B->ctl, mode,
                                                                  vp(B, xv), ncomp);
    BPOST(B);
    return 0;
}

template <typename T>
void set_coarse_ops(fhd_batch* B, const double* eta, double theta) {
    // theta and the viscosities into the coarse-kernel operators
    StagCoarseArgs<T>* sa = reinterpret_cast<StagCoarseArgs<T>*>(B->sargs_h.data());
    for (int b = 0; b < B->nbox; b++)
        for (int q = 0; q < sa[b].nlev; q++) {
            sa[b].A[q].alpha_scale = (T)theta;
            sa[b].A[q].beta0 = (T)eta[b];
        }
    cudaMemcpy(B->sargs, sa, B->sargs_h.size(), cudaMemcpyHostToDevice);
}

// batched GMRES (gmres.f90:32-491) on vectors b (V_B) and x (V_X) with the
// per-box absolute tolerances in B->dabs.  Three fixed launch sequences:
//   init  -- control reset, |M^-1 b| and |b|, x = 0 where b is below the
//            absolute tolerance;
//   outer -- b - A x, its preconditioned norm, the stopping tests, and the
//            number of boxes still running copied to pinned host memory;
//   inner -- V_0 = r/|r|, the m Arnoldi slots (masked per box), the update
//            of x.
// Each is captured once as a CUDA graph (per theta: it is a kernel argument)
// and replayed; the host reads the live count once per cycle.
GParams gparams(const fhd_batch* B) {
    GParams P;
    P.rel_tol = B->p.gmres_rel_tol;
    P.wp = B->p.p_norm_weight;
    P.m = B->m;
    P.max_iter = B->p.gmres_max_iter;
    P.min_iter = B->p.gmres_min_iter;
    P.max_outer = B->p.gmres_max_outer;
    return P;
}

template <typename T>
int gmres_init(fhd_batch* B, double theta) {
    cudaStream_t st = B->stream;
    const int nb = B->nbox, n0 = B->ntab0;
    const double wp2 = B->p.p_norm_weight * B->p.p_norm_weight;
    kb_ctl_reset<<<(nb * 32 + 255) / 256, 256, 0, st>>>(nb, B->ctl, B->deta, B->dabs);
    BPOST(B);
    int rc;
    if ((rc = precon<T>(B, V_B, V_TMP, M_ALL, theta))) return rc;
    kb_dot<<<tgrid(B, kb_dot, n0), TB, 0, st>>>(B->tab0, n0, B->dlev_s, B->ctl, M_ALL, vp(B, V_TMP), vp(B, V_TMP),
                                               wp2, B->part);
    BPOST(B);
    if ((rc = seg(B, M_ALL, 0))) return rc;
    kb_dot<<<tgrid(B, kb_dot, n0), TB, 0, st>>>(B->tab0, n0, B->dlev_s, B->ctl, M_ALL, vp(B, V_B), vp(B, V_B), wp2,
                                               B->part);
    BPOST(B);
    if ((rc = seg(B, M_ALL, 1))) return rc;
    kb_ctl_init<<<(nb + 127) / 128, 128, 0, st>>>(nb, B->ctl);
    BPOST(B);
    kb_zero_x<<<tgrid(B, kb_zero_x, n0), TB, 0, st>>>(B->tab0, n0, B->dlev_s, B->ctl, vp(B, V_X));
    BPOST(B);
    return 0;
}

template <typename T>
int gmres_outer(fhd_batch* B, double theta) {
    cudaStream_t st = B->stream;
    const int nb = B->nbox, n0 = B->ntab0, cb = (nb + 127) / 128;
    const double wp2 = B->p.p_norm_weight * B->p.p_norm_weight;
    int rc;
    // tmp = b - A x, r = M^-1 tmp, the stopping tests
    kb_stokes_apply<<<tgrid(B, kb_stokes_apply, n0), TB, 0, st>>>(B->tab0, n0, B->dlev_s, B->ctl, M_LIVE,
                                                                   vp(B, V_X), vp(B, V_B), vp(B, V_TMP), 1,
                                                                   B->ones64, theta);
    BPOST(B);
    kb_dot<<<tgrid(B, kb_dot, n0), TB, 0, st>>>(B->tab0, n0, B->dlev_s, B->ctl, M_LIVE, vp(B, V_TMP), vp(B, V_TMP),
                                               wp2, B->part);
    BPOST(B);
    if ((rc = seg(B, M_LIVE, 0))) return rc;
    if ((rc = precon<T>(B, V_TMP, V_R, M_LIVE, theta))) return rc;
    kb_dot<<<tgrid(B, kb_dot, n0), TB, 0, st>>>(B->tab0, n0, B->dlev_s, B->ctl, M_LIVE, vp(B, V_R), vp(B, V_R), wp2,
                                               B->part);
    BPOST(B);
    if ((rc = seg(B, M_LIVE, 1))) return rc;
    kb_ctl_outer<<<cb, 128, 0, st>>>(nb, B->ctl, gparams(B));
    BPOST(B);
    // boxes still running
    if (cudaMemsetAsync(B->dlive, 0, sizeof(int), st) != cudaSuccess) return FHD_ERR_CUDA;
    kb_count_live<<<cb, 128, 0, st>>>(nb, B->ctl, B->dlive);
    BPOST(B);
    if (cudaMemcpyAsync(B->hlive, B->dlive, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return FHD_ERR_CUDA;
    return 0;
}

template <typename T>
int gmres_inner(fhd_batch* B, double theta) {
    cudaStream_t st = B->stream;
    const int nb = B->nbox, m = B->m, n0 = B->ntab0, cb = (nb + 127) / 128;
    const double wp2 = B->p.p_norm_weight * B->p.p_norm_weight;
    const GParams P = gparams(B);
    int rc;
    // V_0 = r / |r|
    kb_scale<<<tgrid(B, kb_scale, n0), TB, 0, st>>>(B->tab0, n0, B->dlev_s, B->ctl, vp(B, V_V0), vp(B, V_R), -1);
    BPOST(B);
    for (int i = 1; i <= m; i++) {
        kb_stokes_apply<<<tgrid(B, kb_stokes_apply, n0), TB, 0, st>>>(B->tab0, n0, B->dlev_s, B->ctl, M_INNER,
                                                                       vp(B, V_V0 + i - 1), vp(B, V_V0 + i - 1),
                                                                       vp(B, V_TMP), 0, B->ones64, theta);
        BPOST(B);
        if ((rc = precon<T>(B, V_TMP, V_W, M_INNER, theta))) return rc;
        for (int k = 1; k <= i; k++) {
            kb_mgs<<<tgrid(B, kb_mgs, n0), TB, 0, st>>>(B->tab0, n0, B->dlev_s, B->ctl, vp(B, V_W),
                                                       k > 1 ? vp(B, V_V0 + k - 2) : nullptr, k - 1,
                                                       vp(B, V_V0 + k - 1), wp2, B->part);
            BPOST(B);
            if ((rc = seg(B, M_INNER, 5 + k))) return rc;
        }
        kb_mgs<<<tgrid(B, kb_mgs, n0), TB, 0, st>>>(B->tab0, n0, B->dlev_s, B->ctl, vp(B, V_W), vp(B, V_V0 + i - 1),
                                                   i, nullptr, wp2, B->part);
        BPOST(B);
        if ((rc = seg(B, M_INNER, 5 + i + 1))) return rc;
        kb_scale<<<tgrid(B, kb_scale, n0), TB, 0, st>>>(B->tab0, n0, B->dlev_s, B->ctl, vp(B, V_V0 + i), vp(B, V_W),
                                                       i + 1);
        BPOST(B);
        kb_ctl_inner<<<cb, 128, 0, st>>>(nb, B->ctl, i, P);
        BPOST(B);
    }
    kb_update_sol<<<tgrid(B, kb_update_sol, n0), TB, 0, st>>>(B->tab0, n0, B->dlev_s, B->ctl, vp(B, V_X),
                                                               vc(B, V_V0, 0), (i64)3 * B->N0, B->N0);
    BPOST(B);
    kb_ctl_clear_pend<<<cb, 128, 0, st>>>(nb, B->ctl);
    BPOST(B);
    return 0;
}

// capture body() on the batch's stream as graph `which`; its kernel count is
// added to the launch counter at every replay instead
template <class F>
int capture(fhd_batch* B, int which, F body) {
    const long long n_before = B->launches;
    if (cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return FHD_ERR_CUDA;
    const int rc = body();
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(B->stream, &g);
    B->gn[which] = B->launches - n_before;
    B->launches = n_before;
    if (rc || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        set_last_error(std::string("batched graph capture: ") + cudaGetErrorString(e));
        return rc ? rc : FHD_ERR_CUDA;
    }
    if (B->gx[which]) cudaGraphExecDestroy(B->gx[which]);
    B->gx[which] = nullptr;
    const cudaError_t ei = cudaGraphInstantiate(&B->gx[which], g, 0);
    cudaGraphDestroy(g);
    return ei == cudaSuccess ? 0 : FHD_ERR_CUDA;
}

int replay(fhd_batch* B, int which) {
    B->launches += B->gn[which];
    return cudaGraphLaunch(B->gx[which], B->stream) == cudaSuccess ? 0 : FHD_ERR_CUDA;
}

template <typename T>
int gmres(fhd_batch* B, double theta) {
    int rc;
    if (!B->g_ok || B->g_theta != theta) {
        B->g_ok = 0;
        if ((rc = capture(B, 0, [&] { return gmres_init<T>(B, theta); }))) return rc;
        if ((rc = capture(B, 1, [&] { return gmres_outer<T>(B, theta); }))) return rc;
        if ((rc = capture(B, 2, [&] { return gmres_inner<T>(B, theta); }))) return rc;
        B->g_ok = 1;
        B->g_theta = theta;
    }
    if ((rc = replay(B, 0))) return rc;
    for (int cycle = 0; cycle <= B->p.gmres_max_outer + 1; cycle++) {
        if ((rc = replay(B, 1))) return rc;
        if (cudaStreamSynchronize(B->stream) != cudaSuccess) return FHD_ERR_CUDA;
        if (*B->hlive == 0) break;
        if ((rc = replay(B, 2))) return rc;
    }
    return 0;
}

int read_stats(fhd_batch* B, fhd_solve_stats* stats, int* worst) {
    std::vector<Ctl> h(B->nbox);
    if (cudaMemcpy(h.data(), B->ctl, sizeof(Ctl) * B->nbox, cudaMemcpyDeviceToHost) != cudaSuccess)
        return FHD_ERR_CUDA;
    *worst = 0;
    for (int b = 0; b < B->nbox; b++) {
        *worst = std::max(*worst, h[b].status);
        if (!stats) continue;
        fhd_solve_stats& S = stats[b];
        memset(&S, 0, sizeof(S));
        S.outer_iters = h[b].iter;
        S.total_iters = h[b].total_iter;
        S.status = h[b].status;
        S.norm_b = h[b].norm_b;
        S.norm_pre_b = h[b].norm_pre_b;
        S.norm_init_resid = h[b].norm_init_resid;
        S.norm_resid = h[b].norm_resid;
        S.norm_resid_Stokes = h[b].norm_resid_Stokes;
        S.norm_init_Stokes = h[b].norm_init_Stokes;
        S.norm_resid_est = h[b].norm_resid_est;
    }
    return 0;
}

}  // namespace

extern "C" {

int fhd_batch_create(int nboxes, const int* n_cells, double dx, const fhd_gmres_params* params, int precision_mode,
                     fhd_batch** out) {
    if (!out || !n_cells || nboxes < 1 || !(dx > 0.0)) return FHD_ERR_BAD_ARG;
    *out = nullptr;
    fhd_gmres_params p;
    if (params) p = *params;
    else fhd_gmres_params_default(&p);
    if (p.precon_type != 1 || p.visc_schur_approx != 0 || p.stag_mg_max_vcycles != 1 || p.mg_max_vcycles != 1 ||
        p.gmres_spatial_order != 2 || p.stag_mg_smoother == 0 || p.scale_factor != 1.0 || p.gmres_max_inner < 1 ||
        p.gmres_max_inner > MAXM) {
        set_last_error("fhd_batch_create: precon_type 1, one V-cycle per multigrid call, the colour smoother, "
                       "scale_factor 1 and gmres_max_inner <= 16 are supported");
        return FHD_ERR_UNSUPPORTED;
    }
    for (int b = 0; b < nboxes; b++)
        if (n_cells[2 * b] < 2 || n_cells[2 * b + 1] < 2) return FHD_ERR_BAD_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return FHD_ERR_NO_DEVICE;
    fhd_batch* B = new fhd_batch();
    B->nbox = nboxes;
    B->prec = precision_mode == FHD_PREC_MIXED ? FHD_PREC_MIXED : FHD_PREC_FP64;
    B->dx = dx;
    B->p = p;
    B->m = p.gmres_max_inner;
    B->nx.resize(nboxes);
    B->ny.resize(nboxes);
    B->nls.resize(nboxes);
    B->nlc.resize(nboxes);
    B->lcs.resize(nboxes);
    B->lcc.resize(nboxes);
    int rc = 0;
    for (int b = 0; b < nboxes && !rc; b++) {
        B->nx[b] = n_cells[2 * b];
        B->ny[b] = n_cells[2 * b + 1];
        B->nls[b] = nlevs(B->nx[b], B->ny[b], p.stag_mg_minwidth);
        B->nlc[b] = nlevs(B->nx[b], B->ny[b], p.mg_minwidth);
        if (B->nls[b] > MAXL || B->nlc[b] > MAXL) rc = FHD_ERR_UNSUPPORTED;
    }
    int dev = 0;
    if (!rc && (cudaGetDevice(&dev) != cudaSuccess ||
                cudaDeviceGetAttribute(&B->sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
                cudaDeviceGetAttribute(&B->smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
                cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking) != cudaSuccess))
        rc = FHD_ERR_CUDA;
    if (!rc) rc = B->prec == FHD_PREC_MIXED ? build<float>(B) : build<double>(B);
    if (rc) {
        if (rc == FHD_ERR_UNSUPPORTED && fhd_last_error()[0] == '\0')
            set_last_error("fhd_batch_create: a box's multigrid does not fit the batched layout");
        fhd_batch_destroy(B);
        return rc;
    }
    *out = B;
    return FHD_OK;
}

int fhd_batch_destroy(fhd_batch* B) {
    if (!B) return FHD_ERR_BAD_ARG;
    if (B->stream) cudaStreamSynchronize(B->stream);
    for (cudaGraphExec_t& g : B->gx)
        if (g) cudaGraphExecDestroy(g);
    for (void* p : B->allocs) cudaFree(p);
    if (B->hlive) cudaFreeHost(B->hlive);
    if (B->stream) cudaStreamDestroy(B->stream);
    delete B;
    return FHD_OK;
}

long long fhd_batch_box_offset(fhd_batch* B, int box) {
    if (!B || box < 0 || box > B->nbox) return FHD_ERR_BAD_ARG;
    long long off = 0;
    for (int b = 0; b < box; b++) off += (long long)B->nx[b] * B->ny[b];
    return off;
}

long long fhd_batch_kernel_launches(fhd_batch* B) { return B ? B->launches : 0; }

int fhd_batch_gmres(fhd_batch* B, const double* const b[3], double* const x[3], const double* eta,
                    double theta_alpha, fhd_solve_stats* stats) {
    if (!B || !b || !x || !eta) return FHD_ERR_BAD_ARG;
    cudaStream_t st = B->stream;
    const size_t bytes = sizeof(double) * (size_t)B->N0;
    for (int c = 0; c < 3; c++) {
        if (!b[c] || !x[c]) return FHD_ERR_BAD_ARG;
        FHD_CUDA_TRY(cudaMemcpyAsync(vc(B, V_B, c), b[c], bytes, cudaMemcpyDeviceToDevice, st));
        FHD_CUDA_TRY(cudaMemcpyAsync(vc(B, V_X, c), x[c], bytes, cudaMemcpyDeviceToDevice, st));
    }
    FHD_CUDA_TRY(cudaMemcpyAsync(B->deta, eta, sizeof(double) * B->nbox, cudaMemcpyHostToDevice, st));
    std::vector<double> abs_tol(B->nbox, B->p.gmres_abs_tol);
    FHD_CUDA_TRY(cudaMemcpyAsync(B->dabs, abs_tol.data(), sizeof(double) * B->nbox, cudaMemcpyHostToDevice, st));
    FHD_CUDA_TRY(cudaStreamSynchronize(st));
    int rc;
    if (B->prec == FHD_PREC_MIXED) {
        set_coarse_ops<float>(B, eta, theta_alpha);
        rc = gmres<float>(B, theta_alpha);
    } else {
        set_coarse_ops<double>(B, eta, theta_alpha);
        rc = gmres<double>(B, theta_alpha);
    }
    if (rc < 0) return rc;
    for (int c = 0; c < 3; c++)
        FHD_CUDA_TRY(cudaMemcpyAsync(x[c], vc(B, V_X, c), bytes, cudaMemcpyDeviceToDevice, st));
    FHD_CUDA_TRY(cudaStreamSynchronize(st));
    int worst = 0;
    if ((rc = read_stats(B, stats, &worst))) return rc;
    return worst;
}

int fhd_batch_overdamped(fhd_batch* B, double* const umac[2], double* pi, const double* eta, const double* kT,
                         double dt, int steps, unsigned long long seed, int step0, int* gmres_iters) {
    if (!B || !umac || !umac[0] || !umac[1] || !pi || !eta || !kT || !(dt > 0.0) || steps < 0) return FHD_ERR_BAD_ARG;
    cudaStream_t st = B->stream;
    const int nb = B->nbox;
    FHD_CUDA_TRY(cudaMemcpyAsync(B->deta, eta, sizeof(double) * nb, cudaMemcpyHostToDevice, st));
    FHD_CUDA_TRY(cudaMemcpyAsync(B->dkT, kT, sizeof(double) * nb, cudaMemcpyHostToDevice, st));
    FHD_CUDA_TRY(cudaMemsetAsync(B->ctl, 0, sizeof(Ctl) * nb, st));
    {
        // the viscosities into the control blocks before the first
        // right-hand side reads them
        std::vector<double> a0(nb, B->p.gmres_abs_tol);
        FHD_CUDA_TRY(cudaMemcpyAsync(B->dabs, a0.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, st));
        kb_ctl_reset<<<(nb * 32 + 255) / 256, 256, 0, st>>>(nb, B->ctl, B->deta, B->dabs);
        if (int r0 = post(B)) return r0;
    }
    FHD_CUDA_TRY(cudaStreamSynchronize(st));
    if (B->prec == FHD_PREC_MIXED) set_coarse_ops<float>(B, eta, 0.0);
    else set_coarse_ops<double>(B, eta, 0.0);
    // the state (u, p) in the solution vector's table: x = (du, dp), b = rhs
    double* const s_ptr[3] = {umac[0], umac[1], pi};
    double** d_s = nullptr;
    FHD_CUDA_TRY(cudaMallocAsync((void**)&d_s, sizeof(double*) * 3, st));
    FHD_CUDA_TRY(cudaMemcpyAsync(d_s, s_ptr, sizeof(double*) * 3, cudaMemcpyHostToDevice, st));
    const size_t bytes = sizeof(double) * (size_t)B->N0;
    const double abs_tol_in = B->p.gmres_abs_tol;
    std::vector<double> base(nb, abs_tol_in);
    int worst = 0, rc = 0;
    for (int s = 0; s < steps && rc >= 0; s++) {
        // two stages (advance_timestep_overdamped.f90:228-246, 480-500):
        // h = dt/2 with stage weights (1, 0), then h = dt with (1, 1)/sqrt 2
        for (int stage = 0; stage < 2 && rc >= 0; stage++) {
            const double h = stage == 0 ? 0.5 * dt : dt;
            StepNoise N;
            N.seed = seed;
            N.step = (uint32_t)(step0 + s);
            N.w[0] = stage == 0 ? 1.0 : 1.0 / std::sqrt(2.0);
            N.w[1] = stage == 0 ? 0.0 : 1.0 / std::sqrt(2.0);
            N.var_fac = 2.0 / (B->dx * B->dx * h);  // variance_coef_mom 1, dV = dx^2 (unit depth)
            if (B->prec == FHD_PREC_MIXED)
                kb_step_rhs<float><<<tgrid(B, kb_step_rhs<float>, B->ntab0), TB, 0, st>>>(B->tab0, B->ntab0, B->dlev_s, B->ctl, d_s, pi, vp(B, V_B),
                                                            vc(B, V_B, 2), B->ones64, B->dkT, N);
            else
                kb_step_rhs<double><<<tgrid(B, kb_step_rhs<double>, B->ntab0), TB, 0, st>>>(B->tab0, B->ntab0, B->dlev_s, B->ctl, d_s, pi, vp(B, V_B),
                                                             vc(B, V_B, 2), B->ones64, B->dkT, N);
            if ((rc = post(B))) break;
            for (int c = 0; c < 3; c++)
                if (cudaMemsetAsync(vc(B, V_X, c), 0, bytes, st) != cudaSuccess) rc = FHD_ERR_CUDA;
            if (stage == 0) {
                if (cudaMemcpyAsync(B->dabs, base.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, st) !=
                    cudaSuccess)
                    rc = FHD_ERR_CUDA;
            } else {
                // the corrector stops at the predictor's preconditioned rhs
                kb_set_abs_tol<<<(nb + 127) / 128, 128, 0, st>>>(nb, B->ctl, B->dabs, abs_tol_in,
                                                                B->p.gmres_rel_tol);
                if (!rc) rc = post(B);
            }
            if (rc) break;
            const int r2 = B->prec == FHD_PREC_MIXED ? gmres<float>(B, 0.0) : gmres<double>(B, 0.0);
            if (r2 < 0) {
                rc = r2;
                break;
            }
            kb_axpy3<<<tgrid(B, kb_axpy3, B->ntab0), TB, 0, st>>>(B->tab0, B->ntab0, B->dlev_s, d_s, vp(B, V_X));
            if ((rc = post(B))) break;
            int w = 0;
            if ((rc = read_stats(B, nullptr, &w))) break;
            worst = std::max(worst, w);
        }
    }
    cudaFreeAsync(d_s, st);
    if (cudaStreamSynchronize(st) != cudaSuccess && rc >= 0) rc = FHD_ERR_CUDA;
    if (rc < 0) return rc;
    if (gmres_iters) {
        std::vector<Ctl> h(nb);
        FHD_CUDA_TRY(cudaMemcpy(h.data(), B->ctl, sizeof(Ctl) * nb, cudaMemcpyDeviceToHost));
        for (int b = 0; b < nb; b++) gmres_iters[b] = h[b].iters_acc;
    }
    return worst;
}

}  // extern "C"
