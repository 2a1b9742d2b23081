// fhd_rb.cuh -- one full red-black Gauss-Seidel smooth per launch (3D).
//
// The reference smooths colour by colour, a ghost exchange between colours
// (stag_mg_solver.f90:360-396 for the staggered smoother with its 2*dim
// colours; the cell-centred red-black smoother of the pressure multigrid
// likewise).  On the GPU a colour sweep reads the whole array to update half
// of it, so two colour launches cost about seven array passes per smooth.
// Here one CTA owns an x-y tile and a run of z planes and marches up z with
// the planes of the tile (plus a ring) in shared memory:
//
//   plane k+3 arrives -> red update of plane k+2 on tile + ring 1,
//                        black update of plane k on the tile, store k-1
//
// The red values a black cell needs at the tile edge are recomputed from the
// ring, so CTAs never exchange data; the smooth is out of place (src -> dst)
// so every CTA reads only pre-smooth values from global memory.  Planes of
// the unknown (ring 2 in y) and of the rhs and the face coefficient (ring 1
// in y) are prefetched RB_AHEAD steps ahead with 16-byte cp.async copies;
// in x every staged row spans [x0 - XR, x0 + TX + XR) with XR = 16 bytes of
// elements, so each copy is one aligned 16-byte chunk (the periodic wrap
// falls on chunk boundaries because nx is a multiple of XR).  Each cell
// update evaluates the same stencil expression as the colour kernels
// (stag_lface_acc / cc_lap_acc) on the same operands; in FP64 the results
// are bit identical to two colour sweeps (and to the oracle).  Per smooth and
// component: one read of src, rhs and the coefficients, one write of dst.
#pragma once
#include "fhd_kernels.cuh"

namespace fhd {

#ifndef FHD_RB_MAXTY
#define FHD_RB_MAXTY 8
#endif
#ifndef FHD_RB_AHEAD
#define FHD_RB_AHEAD 2
#endif
constexpr int RB_MAXTY = FHD_RB_MAXTY;      // tile rows; the CTA has TY+1 warps
constexpr int RB_MAXTHREADS = 32 * (RB_MAXTY + 1);
constexpr int RB_AHEAD = FHD_RB_AHEAD;      // prefetch distance in planes
constexpr int RB_NPH = 5 + RB_AHEAD;        // unknown planes k-1 .. k+3+AHEAD
constexpr int RB_NCF = 3 + RB_AHEAD;        // coefficient planes k .. k+2+AHEAD
constexpr int RB_MAXTX = 64;
constexpr int RB_CHUNKS = 3;                // 16-byte copies per thread per plane

// geometry of the row-tile smoother (fhd_rbx.cuh: rbx_geom)
struct RBXGeom {
    int TY;       // tile rows (divides ny)
    int KZ;       // plane steps of the longest CTA stretch
    int tiles_y;
    int chunks;   // CTAs of the launch (k_stag_rbx: stretches of the work)
    int rows;     // TY + 4 staged unknown rows
    int crows;    // TY + 2 staged coefficient rows
    size_t smem;  // bytes of dynamic shared memory
    int ahead;    // stages in flight beyond the one awaited
    int per_sm;   // resident CTAs per SM the z-run split assumes
    int threads;  // compute threads (256 or 512)
};

struct RBGeom {
    int TX, TY;        // tile interior (TX a multiple of XR, TY even)
    int KZ;            // planes per CTA (divides nz)
    int tiles_x, tiles_y, chunks;
    int XR;            // x margin = elements per 16-byte chunk
    int W;             // staged row length TX + 2 XR
    int rows, crows;   // TY + 4 unknown rows, TY + 2 coefficient rows
    int threads;       // 32 (TY + 1)
};

inline int largest_divisor_le(int n, int cap, int mult) {
    for (int t = cap - cap % mult; t >= mult; t -= mult)
        if (n % t == 0) return t;
    return 0;
}

// tile geometry for a level; false when the level cannot use the fused
// smoother (2D, an odd extent, or nx not a multiple of 16 bytes)
// tx, ty > 0 ask for that tile (the autotuner's candidates); 0 takes the
// widest and tallest tile that divides the level
inline bool rb_geom(const Grid& g, int ncomp, int elem_bytes, RBGeom& G, int tx = 0, int ty = 0) {
    if (g.dim != 3) return false;
    for (int d = 0; d < 3; d++)
        if (g.n[d] < 2 || (g.n[d] & 1)) return false;
    G.XR = 16 / elem_bytes;
    if (g.n[0] % G.XR) return false;
    const int mx = G.XR < 2 ? 2 : G.XR;
    G.TX = largest_divisor_le(g.n[0], RB_MAXTX, mx);
    G.TY = largest_divisor_le(g.n[1], RB_MAXTY, 2);
    if (tx > 0) G.TX = (tx <= RB_MAXTX && tx % mx == 0 && g.n[0] % tx == 0) ? tx : 0;
    if (ty > 0) G.TY = (ty <= RB_MAXTY && ty % 2 == 0 && g.n[1] % ty == 0) ? ty : 0;
    if (!G.TX || !G.TY) return false;
    G.tiles_x = g.n[0] / G.TX;
    G.tiles_y = g.n[1] / G.TY;
    // z-run length: long runs amortise the prologue; split until about two
    // waves of CTAs exist
    const long target = 2L * 148 * 4;
    int kz = g.n[2];
    while ((kz & 1) == 0 && kz > 8 && (long)G.tiles_x * G.tiles_y * ncomp * (g.n[2] / kz) < target) kz /= 2;
    G.KZ = kz;
    G.chunks = g.n[2] / kz;
    G.W = G.TX + 2 * G.XR;
    G.rows = G.TY + 4;
    G.crows = G.TY + 2;
    G.threads = 32 * (G.TY + 1);
    const int cw = G.W / G.XR;
    if (G.rows * cw > RB_CHUNKS * G.threads || G.crows * cw > RB_CHUNKS * G.threads) return false;
    if (G.TX * G.TY / G.XR > G.threads) return false;  // one 16-byte store per thread
    return true;
}

// Where the fused smooth pays: measured on B200 (FP32, one smooth of three
// components), fused vs two colour launches per component: 256^3 551 vs
// 357 us, 128^3 106 vs 62 us, 64^3 26 vs 25 us, 32^3 and below ~19 vs
// ~24 us.  Large levels stay on the colour kernels; the fused launch serves
// the latency-bound coarse levels.
#ifndef FHD_RB_MAX_CELLS
#define FHD_RB_MAX_CELLS (64L * 64 * 64)
#endif
constexpr long RB_MAX_CELLS = FHD_RB_MAX_CELLS;
inline bool rb_use(const Grid& g) { return g.nc <= RB_MAX_CELLS; }

template <typename T>
inline size_t rb_smem(const RBGeom& G, int ncoef) {
    return sizeof(T) * ((size_t)RB_NPH * G.W * G.rows + (size_t)ncoef * RB_NCF * G.W * G.crows);
}

// 16-byte aligned device pointers (the staged copies are 16-byte chunks)
inline bool rb_aligned(const void* p) { return ((uintptr_t)p & 15) == 0; }

// ---------------------------------------------------------------------
// asynchronous global -> shared copies (sm_80+ cp.async, L2 only)
// ---------------------------------------------------------------------
__device__ __forceinline__ void cp_async16(void* s, const void* g) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(s);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

__device__ __forceinline__ int pmod(int p, int m) { return (p % m + m) % m; }

// Per-thread copy plan of one staged plane: for each of its chunks, the
// in-plane global element offset (wrapped periodically, the same for every
// z) and the shared-memory element offset; -1 = no chunk.
struct ChunkPlan {
    int goff[RB_CHUNKS];
    int soff[RB_CHUNKS];
};

__device__ __forceinline__ void plan_chunks(ChunkPlan& pl, const RBGeom& G, int x0, int y0, int ring, int nrows,
                                            int nx, int ny, int tid) {
    const int cw = G.W / G.XR;
#pragma unroll
    for (int m = 0; m < RB_CHUNKS; m++) {
        const int e = tid + G.threads * m;
        const int r = e / cw, cx = e - r * cw;
        const bool ok = e < nrows * cw;
        pl.goff[m] = ok ? wrapc(y0 + r - ring, ny) * nx + wrapc(x0 - G.XR + cx * G.XR, nx) : 0;
        pl.soff[m] = ok ? e * G.XR : -1;
    }
}

template <typename T>
__device__ __forceinline__ void issue_chunks(const ChunkPlan& pl, T* s, const T* gplane) {
#pragma unroll
    for (int m = 0; m < RB_CHUNKS; m++)
        if (pl.soff[m] >= 0) cp_async16(s + pl.soff[m], gplane + pl.goff[m]);
}

// pointers of one row of the march, all indexed by lx (-XR <= lx < TX+XR):
// plane p rows ly-1, ly, ly+1, planes p-1 and p+1 row ly, coefficient rows
template <typename T, int NCOEF>
struct RBRow {
    T* r0;
    const T *rm, *rp, *zm, *zp;
    const T* cf[NCOEF > 0 ? NCOEF : 1];
    // unknown at unit offset (a, b, c) from (lx, ly, p); the offsets are
    // compile-time constants at every call, so this is one shared load
    __device__ __forceinline__ T at(int lx, int a, int b, int c) const {
        return c < 0 ? zm[lx] : c > 0 ? zp[lx] : b < 0 ? rm[lx] : b > 0 ? rp[lx] : r0[lx + a];
    }
};

template <typename T, int NCOEF>
struct RBTile {
    T* ph;  // RB_NPH unknown planes (W x rows)
    T* cf;  // NCOEF x RB_NCF coefficient planes (W x crows)
    int W, plane, cplane;
    int x0, y0, nx, ny, nz;
    __device__ __forceinline__ T* pbuf(int p) const { return ph + pmod(p, RB_NPH) * plane; }
    __device__ __forceinline__ T* cbuf(int a, int p) const { return cf + (a * RB_NCF + pmod(p, RB_NCF)) * cplane; }
    __device__ __forceinline__ CellF cell(int lx, int ly, int p) const {
        CellF P;
        P.set(nx, ny, nz, wrapc(x0 + lx, nx), wrapc(y0 + ly, ny), wrapc(p, nz));
        return P;
    }
};

// The march of one CTA over planes k0 .. k0+KZ-1.  upd(lx, ly, p, row)
// updates cell (lx, ly) of plane p in shared memory.  Parity 0 (red) is
// swept first, as colour 1 of the reference.  Step k, after one barrier:
//
//   store(k-1), black(k), red(k+2)
//
// black(k) needs red(k-1..k+1), finished before the barrier; red(k+2) reads
// only black cells of planes k+1..k+3, which no black update of this step
// touches; store(k-1) reads a finished plane.  Warp w < TY takes black row w
// and red row w, warp TY the red ring rows -1 and TY and the red cells of
// ring columns -1 / TX, so every warp carries two rows.  coef[a]: the staged
// coefficient arrays.
template <typename T, int NCOEF, class Upd>
__device__ __forceinline__ void rb_march(const RBGeom& G, const RBTile<T, NCOEF>& t, const T* __restrict__ src,
                                         T* __restrict__ dst, const T* const* coef, int k0, Upd upd) {
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
    const i64 nxy = (i64)t.nx * t.ny;
    ChunkPlan pp, pc;
    plan_chunks(pp, G, t.x0, t.y0, 2, G.rows, t.nx, t.ny, tid);
    plan_chunks(pc, G, t.x0, t.y0, 1, G.crows, t.nx, t.ny, tid);
    const int kend = k0 + G.KZ;
    auto issue_ph = [&](int p) {
        if (p <= kend + 1) issue_chunks(pp, t.pbuf(p), src + (i64)wrapc(p, t.nz) * nxy);
    };
    auto issue_cf = [&](int p) {
        if (p <= kend)
#pragma unroll
            for (int a = 0; a < NCOEF; a++) issue_chunks(pc, t.cbuf(a, p), coef[a] + (i64)wrapc(p, t.nz) * nxy);
    };
    const int W = G.W, XR = G.XR;
    // the unknown planes p-1, p, p+1 and the coefficient planes p of one
    // plane's update
    struct Planes {
        T *m, *c, *p;
        T* cf[NCOEF > 0 ? NCOEF : 1];
    };
    auto planes_at = [&](int sm, int sc, int sp, int scf) {
        Planes q;
        q.m = t.ph + sm * t.plane;
        q.c = t.ph + sc * t.plane;
        q.p = t.ph + sp * t.plane;
#pragma unroll
        for (int a = 0; a < NCOEF; a++) q.cf[a] = t.cf + (a * RB_NCF + scf) * t.cplane;
        return q;
    };
    auto planes_of = [&](int p) {
        return planes_at(pmod(p - 1, RB_NPH), pmod(p, RB_NPH), pmod(p + 1, RB_NPH), pmod(p, RB_NCF));
    };
    auto row = [&](const Planes& q, int ly) {
        RBRow<T, NCOEF> R;
        const int base = (ly + 2) * W + XR;
        R.r0 = q.c + base;
        R.rm = R.r0 - W;
        R.rp = R.r0 + W;
        R.zm = q.m + base;
        R.zp = q.p + base;
#pragma unroll
        for (int a = 0; a < NCOEF; a++) R.cf[a] = q.cf[a] + (ly + 1) * W + XR;
        return R;
    };
    const int hx = G.TX >> 1;  // cells of one colour per tile row
    // one row of colour par (0 red, 1 black) of plane p, over [0, TX)
    auto sweep_row = [&](const Planes& q, int p, int ly, int par) {
        const RBRow<T, NCOEF> R = row(q, ly);
        const int s = (t.x0 + t.y0 + ly + p + par) & 1;
        for (int h = tx; h < hx; h += 32) upd(s + 2 * h, ly, p, R);
    };
    // red of plane p on the tile and ring 1 (corners excluded)
    auto red_by_warp = [&](const Planes& q, int p) {
        if (ty < G.TY) {
            sweep_row(q, p, ty, 0);
        } else {
            sweep_row(q, p, -1, 0);
            sweep_row(q, p, G.TY, 0);
            if (tx < G.TY) {
                const int ly = tx;
                upd(((t.x0 - 1 + t.y0 + ly + p) & 1) ? G.TX : -1, ly, p, row(q, ly));
            }
        }
    };
    // 16-byte vector store of the finished plane p
    auto store = [&](int p, const T* buf) {
        const int vx = G.TX / XR;  // vectors per row
        if (tid < vx * G.TY) {
            const int r = tid / vx, c = (tid - r * vx) * XR;
            const uint4 v = *reinterpret_cast<const uint4*>(buf + (r + 2) * W + XR + c);
            *reinterpret_cast<uint4*>(dst + (i64)p * nxy + (i64)(t.y0 + r) * t.nx + t.x0 + c) = v;
        }
    };
    // group 0: unknown planes k0-2 .. k0+2, coefficients k0-1 .. k0+1;
    // group j = 1..AHEAD: unknown plane k0+2+j, coefficients k0+1+j
    for (int p = k0 - 2; p <= k0 + 2; p++) issue_ph(p);
    for (int p = k0 - 1; p <= k0 + 1; p++) issue_cf(p);
    cp_async_commit();
#pragma unroll
    for (int j = 1; j <= RB_AHEAD; j++) {
        issue_ph(k0 + 2 + j);
        issue_cf(k0 + 1 + j);
        cp_async_commit();
    }
    cp_async_wait<RB_AHEAD>();
    __syncthreads();
    // red of k0-1 .. k0+1 read only black cells, which none of them writes
    red_by_warp(planes_of(k0 - 1), k0 - 1);
    red_by_warp(planes_of(k0), k0);
    red_by_warp(planes_of(k0 + 1), k0 + 1);
    // ring slots of unknown plane k-1 and coefficient plane k, advanced by
    // one per step (no modulo in the march)
    int sm = pmod(k0 - 1, RB_NPH), sc = pmod(k0, RB_NCF);
    auto ring = [](int s, int d, int n) { return s + d >= n ? s + d - n : s + d; };
    for (int k = k0; k < kend; k++) {
        // unknown plane k+3 and coefficient plane k+2 are in the group
        // committed AHEAD groups before the newest
        cp_async_wait<RB_AHEAD - 1>();
        __syncthreads();
        // refill the buffers of unknown plane k+3+AHEAD-NPH = k-2 and
        // coefficient plane k+2+AHEAD-NCF = k-1, unused from this step on
        issue_ph(k + 3 + RB_AHEAD);
        issue_cf(k + 2 + RB_AHEAD);
        cp_async_commit();
        const int s0 = ring(sm, 1, RB_NPH), s1 = ring(sm, 2, RB_NPH);
        if (k > k0) store(k - 1, t.ph + sm * t.plane);
        if (ty < G.TY) sweep_row(planes_at(sm, s0, s1, sc), k, ty, 1);
        if (k + 2 <= kend)
            red_by_warp(planes_at(s1, ring(sm, 3, RB_NPH), ring(sm, 4, RB_NPH), ring(sc, 2, RB_NCF)), k + 2);
        sm = s0;
        sc = ring(sc, 1, RB_NCF);
    }
    cp_async_wait<0>();
    __syncthreads();
    store(kend - 1, t.pbuf(kend - 1));
}

// x / d of the update: the quotient of the colour kernels (sm_quot)
template <typename T>
__device__ __forceinline__ T rb_quot(T x, T d) {
    return sm_quot(x, d);
}

template <typename T>
struct RBArgs {
    const T* src[3];
    T* dst[3];
    const T* rhs[3];
    const T* oth[3];  // current values of the other components (coupled visc)
};

template <typename T, int NCOEF>
__device__ __forceinline__ RBTile<T, NCOEF> rb_tile(const Grid& g, const RBGeom& G, unsigned char* raw) {
    RBTile<T, NCOEF> t;
    t.ph = reinterpret_cast<T*>(raw);
    t.W = G.W;
    t.plane = G.W * G.rows;
    t.cplane = G.W * G.crows;
    t.cf = t.ph + RB_NPH * t.plane;
    t.x0 = (blockIdx.x % G.tiles_x) * G.TX;
    t.y0 = (blockIdx.x / G.tiles_x) * G.TY;
    t.nx = g.n[0]; t.ny = g.n[1]; t.nz = g.n[2];
    return t;
}

// staged coefficients of the staggered smoother: 0 = alpha[C], 1 = rhs[C]
template <typename T, int VISC, int C>
__device__ __forceinline__ void stag_rb_run(const Grid& g, const RBGeom& G, const StagOp<T>& A, const RBArgs<T>& R,
                                            T omega, unsigned char* raw) {
    const RBTile<T, 2> t = rb_tile<T, 2>(g, G, raw);
    const T* const* oth = R.oth;
    const T* coef[2] = {A.alpha[C], R.rhs[C]};
    rb_march<T, 2>(G, t, R.src[C], R.dst[C], coef, blockIdx.y * G.KZ,
                   [&](int lx, int ly, int p, const RBRow<T, 2>& Rw) {
                       const CellF P = t.cell(lx, ly, p);
                       auto own = [&](int a, int b, int c) { return Rw.at(lx, a, b, c); };
                       auto othf = [&](int d, int a, int b, int c) { return ld(oth[d], P.id(a, b, c)); };
                       auto alp = [&]() { return Rw.cf[0][lx]; };
                       T dg;
                       const T L = stag_lface_acc<T, 3, VISC, C>(A, P, own, othf, alp, dg);
                       T& v = Rw.r0[lx];
                       v = v + rb_quot(omega * (Rw.cf[1][lx] - L), dg);
                   });
}

// One full smooth (both colours) of the staggered operator.  CFIX < 0: the
// component is blockIdx.z (uncoupled |visc_type| = 1, all components in one
// launch); otherwise the one component CFIX.
template <typename T, int VISC, int CFIX>
__global__ void __launch_bounds__(RB_MAXTHREADS) k_stag_rb(Grid g, RBGeom G, StagOp<T> A, RBArgs<T> R, T omega) {
    extern __shared__ __align__(16) unsigned char rb_smraw[];
    // the constant viscosity of visc_type > 0, loaded once (the staging
    // asm clobbers memory, which would force a reload per row)
    if constexpr (VISC > 0) {
        if (!A.beta0_set) {
            A.beta0 = A.beta[0];
            A.beta0_set = 1;
        }
    }
    if constexpr (CFIX >= 0) {
        stag_rb_run<T, VISC, CFIX>(g, G, A, R, omega, rb_smraw);
    } else {
        const int c = blockIdx.z;
        if (c == 0) stag_rb_run<T, VISC, 0>(g, G, A, R, omega, rb_smraw);
        else if (c == 1) stag_rb_run<T, VISC, 1>(g, G, A, R, omega, rb_smraw);
        else stag_rb_run<T, VISC, 2>(g, G, A, R, omega, rb_smraw);
    }
}

// One full red-black smooth of the cell-centred operator D a G (3D); the
// rhs is staged, the face coefficients are read through the cache.
template <typename T>
__global__ void __launch_bounds__(RB_MAXTHREADS) k_cc_rb(Grid g, RBGeom G, CCOp<T> A, const T* __restrict__ src,
                                                      T* __restrict__ dst, const T* __restrict__ rhs) {
    extern __shared__ __align__(16) unsigned char rb_smraw[];
    const RBTile<T, 1> t = rb_tile<T, 1>(g, G, rb_smraw);
    const T* coef[1] = {rhs};
    rb_march<T, 1>(G, t, src, dst, coef, blockIdx.y * G.KZ, [&](int lx, int ly, int p, const RBRow<T, 1>& Rw) {
        const CellF P = t.cell(lx, ly, p);
        auto ph = [&](int a, int b, int c) { return Rw.at(lx, a, b, c); };
        T dg;
        const T L = cc_lap_acc<T, 3>(A, P, ph, dg);
        T& v = Rw.r0[lx];
        v = v + rb_quot(Rw.cf[0][lx] - L, dg);
    });
}

}  // namespace fhd
