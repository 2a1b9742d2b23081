// fhd_rbx.cuh -- one full red-black smooth per launch on the large levels
// of the FP32 staggered multigrid, constant-coefficient operator
// (visc_type 1), 3D, x extent of 64 to 256 cells.
//
// The same z-march as the tiled fused smoother (fhd_rb.cuh: red update of
// plane k+2 on the tile and a ring, black update of plane k, store of plane
// k-1, out of place src -> dst), with the tile widened to whole x rows so
// that the periodic x wrap stays inside shared memory and no x ring is
// recomputed, and with the planes staged by the bulk-copy engine:
//
//   * a producer warp copies the staged rows of a plane (unknown rows
//     y0-2 .. y0+TY+1, diagonal and rhs rows y0-1 .. y0+TY) with 1D
//     cp.async.bulk copies, one per array and contiguous run of rows (the
//     periodic y wrap splits a run), completing on the stage's mbarrier;
//   * eight compute warps update four to five cells per thread and plane
//     step, every update one evaluation of stag_lface_acc on shared memory
//     (the same expression as the colour kernels and the oracle);
//   * the finished plane's TY interior rows, contiguous in shared and in
//     global memory, are written by the compute threads with 16-byte
//     stores at the next plane step.  A bulk store from the producer warp
//     queued behind that step's loads, and the producer then waited for it
//     before refilling the slot; the producer warp now only loads.
//
// Every mbarrier wait is bounded; a wait that runs out sets *err, and the
// CTA leaves together (after its copies in flight have landed, again with a
// bound) through the step barrier's reduction.
#pragma once
#include <type_traits>

#include "fhd_kernels.cuh"

namespace fhd {

constexpr int RBX_THREADS = 256;  // compute threads (the wide form: 512)
// stages in flight beyond the one awaited (the rings then hold unknown
// planes k-1 .. k+3 and coefficient planes k .. k+2 plus these)
constexpr int RBX_AHEAD = 3;
constexpr int RBX_MAXNX = 256;
constexpr long RBX_SPIN = 1L << 22;     // try_wait polls before a wait gives up
constexpr int RBX_MINRUN = 4;           // shortest z-run of a (tile, component) item
// a thread updates the cells of one x column on rows gr, gr + RG, ..: with
// RG = RBX_THREADS / (nx / 2) its rows lie RBX_ROWSTEP elements apart for
// every nx, at most RBX_MAXR of them per sweep
constexpr int RBX_ROWSTEP = 2 * RBX_THREADS;
constexpr int RBX_MAXR = 5;
// the block: RBX_THREADS compute threads and one producer warp
constexpr int RBX_BLOCK = RBX_THREADS + 32;
// rows per thread and sweep for nt compute threads: 5 with 256, 3 with 512
// (twice the warps to hide the update chains, each taking fewer rows)
constexpr int rbx_maxr(int nt) { return nt == 256 ? 5 : 3; }
// Every thread evaluates RBX_MAXR rows per sweep and stores only those of
// the tile.  The reads of the others stay below RBX_MAXR * RBX_ROWSTEP +
// 2 nx elements from the start of an unknown plane slot and below
// RBX_MAXR * RBX_ROWSTEP from the start of a coefficient slot; shared memory
// holds the coefficient ring, then the unknown ring, then a pad that covers
// the last unknown slot's overrun.
inline int rbx_pad(int nx, int rows, int nt = RBX_THREADS) {
    const int over = rbx_maxr(nt) * 2 * nt + 2 * nx - rows * nx;
    return (over > 0 ? over : 0) + 32;
}
// ahead: stages in flight beyond the one awaited (RBX_AHEAD, or 1 for the
// variant that fits two CTAs on an SM); nt: compute threads
inline size_t rbx_smem_bytes(int nx, int ty, int ahead = RBX_AHEAD, int nt = RBX_THREADS) {
    return 64 + sizeof(float) * ((size_t)(3 + ahead) * 2 * (ty + 2) * nx + (size_t)(5 + ahead) * (ty + 4) * nx +
                                 rbx_pad(nx, ty + 4, nt));
}

// ---------------------------------------------------------------------
// mbarrier and bulk-copy primitives (sm_90+ PTX, no cluster multicast)
// ---------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* b, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* b, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(b)), "r"(bytes)
                 : "memory");
}
// true once the phase of parity `parity` has completed
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* b, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait: false when the phase did not complete within RBX_SPIN polls
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* b, unsigned parity) {
    for (long i = 0; i < RBX_SPIN; i++)
        if (mbar_try_wait(b, parity)) return true;
    return false;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* b) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(b))
                 : "memory");
}
// generic-proxy shared-memory accesses ordered before later async-proxy ones
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// ---------------------------------------------------------------------
// the kernel
// ---------------------------------------------------------------------
// Cut b of P over the work of `items` items of nz planes each, flattened
// item by item: W * b / P, moved to the item's edge when it would leave a
// run shorter than RBX_MINRUN planes.  The move is non-decreasing in the
// cut, so the cuts stay ordered.  With P = items * c the cuts are the edges
// of c equal z-runs per item.
__host__ __device__ inline long rbx_cut(long items, int nz, long b, long P) {
    const long W = items * nz;
    long x = W * b / P;
    const long k = x % nz;
    if (k != 0 && k < RBX_MINRUN) x -= k;
    else if (k != 0 && nz - k < RBX_MINRUN) x += nz - k;
    return x;
}
struct RBXArgs {
    const float* src[3];
    float* dst[3];
    const float* rhs[3];
    const float* diag[3];  // the visc_type 1 diagonal (stag_diag1), staged in place of alpha
    unsigned* err;
};

// One z-run of one (tile, component) item: planes k0 .. kend-1 of tile row
// tile_y.  qb: stages this CTA has issued before the run (its earlier runs),
// so that every mbarrier keeps counting its phases across runs; nstages
// returns the run's stage count.  False when a staging wait timed out.
template <int C, int AH, int NT>
__device__ __forceinline__ bool rbx_run(const Grid& g, const RBXGeom& G, const StagOp<float>& A0, const RBXArgs& R,
                                        float omega, unsigned char* raw, int tile_y, int k0, int kend, int qb,
                                        int& nstages) {
    // the constant viscosity, loaded once: every asm statement below clobbers
    // memory, which would make each sweep reload it from global memory
    StagOp<float> A = A0;
    if (!A.beta0_set) {
        A.beta0 = A0.beta[0];
        A.beta0_set = 1;
    }
    const float bq = A.beta0 * A.q;
    constexpr int NPH = 5 + AH;  // unknown planes k-1 .. k+3 + in flight
    constexpr int NCF = 3 + AH;  // coefficient planes k .. k+2 + in flight
    constexpr int MR = rbx_maxr(NT);  // rows per thread and red sweep
    constexpr int ROWSTEP = 2 * NT;   // elements between a thread's rows
    const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
    const int TY = G.TY, rows = G.rows, crows = G.crows;
    const int tid = threadIdx.x;
    const i64 nxy = (i64)nx * ny;
    const int y0 = tile_y * TY;
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(raw);
    const int plane = rows * nx, cplane = crows * nx;
    float* cf = reinterpret_cast<float*>(raw + 64);  // [slot][0 diagonal, 1 rhs][crows][nx]
    float* ph = cf + NCF * 2 * cplane;          // [slot][rows][nx]
    const float* src = R.src[C];
    float* dst = R.dst[C];
    const float* diag = R.diag[C];
    const float* rhs = R.rhs[C];
    // stage j = unknown plane j (always) + coefficient plane j-1 (for
    // j >= k0); q = j - (k0 - 2) counts the stages of this CTA from 0
    const int qend = kend + 1 - (k0 - 2);  // last stage index
    // stage q issued by the producer warp: lane 0 arms the barrier with the
    // stage's bytes, then lane 0 copies the unknown rows, lanes 1 and 2 the
    // diagonal and rhs rows.  A tile's rows are consecutive in global memory
    // except across the periodic y wrap, so each array goes as one to three
    // contiguous copies.
    auto issue = [&](int q) {
        const int lane = tid - NT;
        const int j = q + k0 - 2;
        const int s = (qb + q) % NPH;
        if (lane == 0) mbar_expect_tx(&bar[s], (unsigned)(sizeof(float) * (plane + (j >= k0 ? 2 * cplane : 0))));
        __syncwarp();
        auto copy = [&](float* sdst, const float* gplane, int nrows, int ring) {
            int r = 0;
            while (r < nrows) {
                const int ys = wrapc(y0 + r - ring, ny);
                const int n = nrows - r < ny - ys ? nrows - r : ny - ys;
                bulk_g2s(sdst + r * nx, gplane + (i64)ys * nx, (unsigned)(sizeof(float) * n * nx), &bar[s]);
                r += n;
            }
        };
        if (lane == 0) copy(ph + s * plane, src + (i64)wrapc(j, nz) * nxy, rows, 2);
        if (j >= k0 && (lane == 1 || lane == 2)) {
            const int cs = pmod(j - 1, NCF);
            const i64 zo = (i64)wrapc(j - 1, nz) * nxy;
            copy(cf + (cs * 2 + lane - 1) * cplane, (lane == 1 ? diag : rhs) + zo, crows, 1);
        }
    };
    // wait for stage q; false on time-out
    auto wait_stage = [&](int q) {
        return mbar_wait_bounded(&bar[(qb + q) % NPH], (unsigned)(((qb + q) / NPH) & 1));
    };

    const int hx = nx >> 1;           // cells of one colour per row
    const int RG = NT / hx;  // rows updated at once
    // a warp takes 16 cells of a colour on each of two adjacent rows: their
    // colour offsets differ by one, so the two half-warps read the even and
    // the odd banks and every shared access is one wavefront
    const int hgrp = hx >> 4;  // 16-cell groups per row
    const int wi = tid >> 5, ln = tid & 31;
    const int h = (wi % hgrp) * 16 + (ln & 15);
    const int gr = 2 * (wi / hgrp) + (ln >> 4);
    int issued = 0;  // stages issued so far (thread 0)
    // update of the cells of parity par on rows ly = ly0 + gr, + RG, .. < ly1
    // of plane p (slots: unknown planes p-1, p, p+1; coefficients p).  RG
    // is even, so the thread's column lx is the same on all its rows.  The
    // RBX_MAXR rows are evaluated without branches and all new values are
    // computed before any is stored (no cell of the colour reads another),
    // so the rows' loads overlap; rows past ly1 read staged or pad memory
    // and are not stored.
    // NR rows per thread (RBX_MAXR - 1 cover the tile rows, RBX_MAXR the
    // tile and its ring);
    // sm / sc / sp: ring slots of unknown planes p-1, p, p+1, scf: the
    // coefficient slot of plane p
    auto sweep = [&](auto NRc, int sm, int sc, int sp, int scf, int p, int par, int ly0, int ly1) {
        constexpr int NR = decltype(NRc)::value;
        const int lyb = ly0 + gr;
        const int lx = 2 * h + ((y0 + lyb + p + par) & 1);
        const int lxm = lx == 0 ? nx - 1 : lx - 1;
        const int lxp = lx == nx - 1 ? 0 : lx + 1;
        const int o = (lyb + 2) * nx, co = (lyb + 1) * nx + lx;
        float* c0 = ph + sc * plane + o;
        const float* zm = ph + sm * plane + o + lx;
        const float* zp = ph + sp * plane + o + lx;
        const float* ca = cf + (scf * 2) * cplane + co;
        const float* cr = ca + cplane;
        float nv[NR];
#pragma unroll
        for (int m = 0; m < NR; m++) {
            const int r = m * ROWSTEP;
            const float* c = c0 + r;
            // ca holds the diagonal (stag_diag1), which stag_lface_acc forms
            // from alpha; stag_l1_f32 is its FP32 visc_type 1 operator
            const float dg = ca[r];
            const float L = stag_l1_f32<float, 3, C>(
                [&](int a, int b, int cz) {
                    return cz < 0   ? zm[r]
                           : cz > 0 ? zp[r]
                           : b < 0  ? c[lx - nx]
                           : b > 0  ? c[lx + nx]
                           : a < 0  ? c[lxm]
                           : a > 0  ? c[lxp]
                                    : c[lx];
                },
                dg, bq);
            nv[m] = c[lx] + sm_quot(omega * (cr[r] - L), dg);
        }
#pragma unroll
        for (int m = 0; m < NR; m++)
            if (lyb + m * RG < ly1) c0[m * ROWSTEP + lx] = nv[m];
    };
    // the TY rows of the finished plane p, contiguous in shared and in global
    // memory, stored by the compute threads
    auto put_plane = [&](int p) {
        const float4* sp = reinterpret_cast<const float4*>(ph + pmod(p - (k0 - 2) + qb, NPH) * plane + 2 * nx);
        float4* gp = reinterpret_cast<float4*>(dst + (i64)p * nxy + (i64)y0 * nx);
        const int n4 = (TY * nx) >> 2;
        for (int e = tid; e < n4; e += NT) gp[e] = sp[e];
    };
    // prologue: stages q = 0 .. 4 (unknown planes k0-2 .. k0+2, coefficient
    // planes k0-1 .. k0+1) and AHEAD more
    const bool producer = tid >= NT;
    const int lead = NT;  // producer lane 0: clean-up after a wait ran out
    if (producer) {
        for (int q = 0; q < 5 + AH && q <= qend; q++) issue(q);
        issued = 5 + AH < qend + 1 ? 5 + AH : qend + 1;
    }
    using RRed = std::integral_constant<int, MR>;
    using RBlack = std::integral_constant<int, MR - 1>;
    auto slot = [&](int p) { return pmod(p - (k0 - 2) + qb, NPH); };
    auto ring = [](int v, int d, int n) { return v + d >= n ? v + d - n : v + d; };
    int sl, scl;
    bool ok = true;
    if (!producer)
        for (int q = 0; q < 5; q++) ok = ok && wait_stage(q);
    if (__syncthreads_or(!ok)) goto fail;
    // red of k0-1 .. k0+1 read only black cells, which none of them writes
    if (!producer)
        for (int p = k0 - 1; p <= k0 + 1; p++) sweep(RRed(), slot(p - 1), slot(p), slot(p + 1), pmod(p, NCF), p, 0, -1, TY + 1);
    // ring slots of unknown plane k-1 and coefficient plane k, advanced by one
    // per step
    sl = slot(k0 - 1);
    scl = pmod(k0, NCF);
    for (int k = k0; k < kend; k++) {
        // this thread's shared-memory accesses of the previous steps are
        // ordered before the bulk copies that refill their slots
        fence_proxy_async();
        if (__syncthreads_or(!ok)) goto fail;
        if (producer) {
            // stage k+3+AHEAD refills the slot of unknown plane k-2 (last
            // read by the black update and the store of step k-1) and the
            // coefficient slot of plane k-1
            const int qn = k + 3 + AH - (k0 - 2);
            if (qn <= qend) {
                issue(qn);
                issued = qn + 1;
            }
            continue;
        }
        // plane k-1 is final since the black update of step k-1
        if (k > k0) put_plane(k - 1);
        // stage k+3: unknown plane k+3, coefficient plane k+2
        if (k + 3 - (k0 - 2) <= qend) ok = wait_stage(k + 3 - (k0 - 2));
        if (!ok) continue;  // leaves at the next barrier
        const int s1 = ring(sl, 1, NPH), s2 = ring(sl, 2, NPH);
        sweep(RBlack(), sl, s1, s2, scl, k, 1, 0, TY);
        if (k + 2 <= kend)
            sweep(RRed(), s2, ring(sl, 3, NPH), ring(sl, 4, NPH), ring(scl, 2, NCF), k + 2, 0, -1, TY + 1);
        sl = s1;
        scl = ring(scl, 1, NCF);
    }
    fence_proxy_async();
    if (__syncthreads_or(!ok)) goto fail;
    if (!producer) {
        put_plane(kend - 1);
        fence_proxy_async();  // before the next run's copies refill the slot
    }
    nstages = qend + 1;
    return true;
fail:
    // a stage did not arrive in time: flag it, let the copies in flight
    // land (bounded) and leave
    if (tid == lead) {
        atomicOr(R.err, 1u);
        // stages before the last NPH issued completed before their
        // barriers were re-armed
        for (int q = issued > NPH ? issued - NPH : 0; q < issued; q++) wait_stage(q);
    }
    return false;
}

// AH stages in flight beyond the one awaited: RBX_AHEAD with one CTA per SM,
// or 1 with two (smaller rings, half the shared memory)
// NT compute threads (256, or 512 in the wide form) and one producer warp
template <int AH, int NT = RBX_THREADS>
__global__ void __launch_bounds__(NT + 32, AH == 1 ? 2 : 1) k_stag_rbx(Grid g, RBXGeom G, StagOp<float> A,
                                                                       RBXArgs R, float omega) {
    extern __shared__ __align__(128) unsigned char rbx_raw[];
    if (threadIdx.x < 5 + AH) mbar_init(reinterpret_cast<unsigned long long*>(rbx_raw) + threadIdx.x, 1);
    if (threadIdx.x == 0) mbar_init_fence();
    __syncthreads();
    // The work is tiles_y * 3 items (tile row, component) of nz planes each,
    // flattened item by item; CTA b takes the stretch between rbx_cut(b)
    // and rbx_cut(b + 1), one z-run per item it touches.
    const int nz = g.n[2];
    const long items = (long)G.tiles_y * 3;
    long s = rbx_cut(items, nz, blockIdx.x, gridDim.x);
    const long e = rbx_cut(items, nz, (long)blockIdx.x + 1, gridDim.x);
    int qb = 0;
    for (bool first = true; s < e; first = false) {
        const long item = s / nz;
        const int k0 = (int)(s % nz);
        const int kend = (int)(e - s < (long)(nz - k0) ? k0 + (e - s) : nz);
        const int comp = (int)(item % 3), tile_y = (int)(item / 3);
        // every thread is done with the staged planes (the previous run's
        // last plane stored from its slot) before this run refills them
        if (!first) __syncthreads();
        int n = 0;
        bool ok;
        if (comp == 0) ok = rbx_run<0, AH, NT>(g, G, A, R, omega, rbx_raw, tile_y, k0, kend, qb, n);
        else if (comp == 1) ok = rbx_run<1, AH, NT>(g, G, A, R, omega, rbx_raw, tile_y, k0, kend, qb, n);
        else ok = rbx_run<2, AH, NT>(g, G, A, R, omega, rbx_raw, tile_y, k0, kend, qb, n);
        if (!ok) return;  // the error word is set; every thread leaves
        qb += n;
        s += kend - k0;
    }
}

// geometry for a level (sms: multiprocessors of the device); false when the
// level cannot use this smoother.  ty > 0 asks for that tile height (the
// autotuner's candidates), 0 for the tallest that fits.
// ahead: RBX_AHEAD, or 1 for two CTAs per SM where smem_sm (shared memory
// of one SM) holds two.
// nt: compute threads, 256 or (with the deep ring) 512.
inline bool rbx_geom(const Grid& g, int sms, size_t smem_max, RBXGeom& G, int ty_req = 0, int ahead = RBX_AHEAD,
                     size_t smem_sm = 0, int nt = RBX_THREADS) {
    if (ahead != RBX_AHEAD && ahead != 1) return false;
    if (nt != RBX_THREADS && !(nt == 512 && ahead == RBX_AHEAD)) return false;
    const int MR = rbx_maxr(nt);
    G.ahead = ahead;
    G.threads = nt;
    if (g.dim != 3) return false;
    const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
    if (nx > RBX_MAXNX || nx < 64 || (nx & (nx - 1)) || (ny & 1) || (nz & 1) || nz < 4) return false;
    const int hx = nx / 2;
    if (nt % hx || hx % 16 || (nt / 32) % (hx / 16)) return false;
    // tallest tile that fits the shared memory of one CTA per SM
    G.TY = 0;
    for (int ty = 32; ty >= 4; ty /= 2) {
        if (ny % ty || (ty_req > 0 && ty != ty_req)) continue;
        const size_t smem = rbx_smem_bytes(nx, ty, ahead, nt);
        if (smem <= smem_max) {
            G.TY = ty;
            G.smem = smem;
            break;
        }
    }
    if (!G.TY) return false;
    // rows per thread and sweep (ring rows included) within MR
    const int RG = nt / hx;
    while (ty_req == 0 && G.TY > 4 && (G.TY + 2 + RG - 1) / RG > MR) G.TY /= 2;
    if ((G.TY + 2 + RG - 1) / RG > MR || (G.TY + RG - 1) / RG > MR - 1 || ny % G.TY) return false;
    G.smem = rbx_smem_bytes(nx, G.TY, ahead, nt);
    if (G.smem > smem_max) return false;
    // resident CTAs per SM (1 KB of each CTA's shared memory is reserved)
    G.per_sm = (ahead == 1 && 2 * (G.smem + 1024) <= smem_sm) ? 2 : 1;
    if (ahead == 1 && G.per_sm == 1) return false;  // the short ring pays only with two CTAs
    G.rows = G.TY + 4;
    G.crows = G.TY + 2;
    G.tiles_y = ny / G.TY;
    // CTAs of the launch: each takes a stretch of the tiles_y * 3 * nz plane
    // steps (rbx_cut).  Candidates: c equal z-runs per item (one item per
    // CTA, in waves when they outnumber the slots), or one CTA per resident
    // slot with stretches that cross item edges.  The cost is the plane steps
    // on the busiest SM, a z-run's prologue counted as five.  With equal
    // z-runs the CTAs of neighbouring row tiles march in step, so the halo
    // rows that both stage are read from DRAM once; stretches desynchronise
    // them and the halo rows are read again (about a quarter more DRAM
    // traffic at 8-row tiles).  Stretches are therefore taken only when they
    // save a tenth of the plane steps.
    const long items = (long)G.tiles_y * 3;
    const long work = items * nz;
    const long slots = (long)sms * G.per_sm;
    auto cost_of = [&](long P) {
        long worst = 0;
        for (long b = 0; b < P; b++) {
            long s0 = rbx_cut(items, nz, b, P);
            const long e0 = rbx_cut(items, nz, b + 1, P);
            long steps = 0;
            while (s0 < e0) {
                const long k0 = s0 % nz;
                const long len = e0 - s0 < nz - k0 ? e0 - s0 : nz - k0;
                steps += len + 5;
                s0 += len;
            }
            worst = steps > worst ? steps : worst;
        }
        return ((P + slots - 1) / slots) * worst;
    };
    long best = -1, bestP = 0;
    auto consider = [&](long P) {
        if (P < 1 || work < P * RBX_MINRUN) return;
        const long c = cost_of(P);
        if (best < 0 || c < best) {
            best = c;
            bestP = P;
        }
    };
    for (int c = 1; c <= nz / 4; c++) consider(items * c);
    if (slots % items != 0 && work >= slots * RBX_MINRUN) {
        const long cs = cost_of(slots);
        if (best < 0 || 10 * cs <= 9 * best) {
            best = cs;
            bestP = slots;
        }
    }
    if (bestP < 1) return false;
    G.chunks = (int)bestP;
    G.KZ = (int)((work + G.chunks - 1) / G.chunks);  // plane steps of the longest stretch
    return true;
}

}  // namespace fhd
