// fhd_kernels.cuh -- sm_100a device kernels of the staggered Stokes solver.
//
// Canonical layout (include/fhd_b200.h): one periodic box, x fastest, face
// array d holds the face on the low-d side of each cell, edges/nodes at the
// low corner.  The periodic wrap replaces the ghost-cell exchange
// (multifab_fill_boundary) that the reference performs after every colour.
//
// All kernels are memory-bound stencils: one thread per cell (or per face of
// a colour), x-contiguous warps for coalesced 128-byte rows, read-only loads
// through the non-coherent path.  Templated on the storage/arithmetic type T
// (double, or float in the mixed-precision preconditioner), the dimension
// and visc_type so the stencil is fully specialised.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace fhd {

typedef long long i64;

struct Grid {
    int dim;
    int n[3];
    i64 nc;
    double dx;
};

__host__ __device__ __forceinline__ int wrapc(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

struct Cell {
    int i, j, k;
    int nx, ny, nz;
    __device__ __forceinline__ i64 id(int di, int dj, int dk) const {
        int a = wrapc(i + di, nx), b = wrapc(j + dj, ny), c = wrapc(k + dk, nz);
        return (i64)a + (i64)nx * ((i64)b + (i64)ny * c);
    }
};

// A cell with its linear index and the six periodic +-1 offsets worked out
// once; id() of a unit offset (compile-time at every call) is then one or
// two additions instead of three wraps and a 64-bit index product.  Gives
// the same indices as Cell.
struct CellF {
    int i, j, k;
    i64 base;
    int oxm, oxp, oym, oyp, ozm, ozp;
    __device__ __forceinline__ void set(const Grid& g, int i_, int j_, int k_) { set(g.n[0], g.n[1], g.n[2], i_, j_, k_); }
    __device__ __forceinline__ void set(int nx, int ny, int nz, int i_, int j_, int k_) {
        i = i_; j = j_; k = k_;
        const int nxy = nx * ny;
        base = (i64)i + (i64)nx * ((i64)j + (i64)ny * k);
        oxm = i == 0 ? nx - 1 : -1;
        oxp = i == nx - 1 ? 1 - nx : 1;
        oym = j == 0 ? (ny - 1) * nx : -nx;
        oyp = j == ny - 1 ? (1 - ny) * nx : nx;
        ozm = k == 0 ? (nz - 1) * nxy : -nxy;
        ozp = k == nz - 1 ? (1 - nz) * nxy : nxy;
    }
    __device__ __forceinline__ i64 id(int di, int dj, int dk) const {
        i64 r = base;
        if (di < 0) r += oxm;
        else if (di > 0) r += oxp;
        if (dj < 0) r += oym;
        else if (dj > 0) r += oyp;
        if (dk < 0) r += ozm;
        else if (dk > 0) r += ozp;
        return r;
    }
};

template <typename T>
__device__ __forceinline__ T ld(const T* p, i64 i) { return __ldg(p + i); }

// x / d of a smoother update: the IEEE quotient in FP64 (bit-identical to
// the oracle); the fast approximate quotient in the FP32 preconditioner,
// where its last-bit error is noise
template <typename T>
__device__ __forceinline__ T sm_quot(T x, T d) {
    if constexpr (sizeof(T) == 4) return __fdividef(x, d);
    else return x / d;
}

// Pointers of one staggered operator level.  alpha is multiplied by
// alpha_scale on the fly (theta_alpha on the finest level).
template <typename T>
struct StagOp {
    const T* alpha[3];
    T alpha_scale;
    const T* beta;
    const T* gamma;
    const T* bed[3];  // 2D: node; 3D: xy, xz, yz
    T q;              // 1/dx^2
    // constant-coefficient operators (visc_type > 0) read beta[0]; a kernel
    // that loaded it once into a register sets beta0_set and beta0
    int beta0_set = 0;
    T beta0 = T(0);
};

template <int DIM>
__host__ __device__ constexpr int edge_of(int c, int d) {
    return DIM == 2 ? 0 : ((c < d ? c : d) == 0 ? ((c > d ? c : d) == 1 ? 0 : 1) : 2);
}

template <int C, int D>
struct Off {
    static constexpr int x = (D == 0), y = (D == 1), z = (D == 2);
};

// visc_type 1: the diagonal alpha_scale alpha + 2 dim beta q (a = alpha_scale
// alpha), and in FP32 the operator given that diagonal, with the transverse
// pairs summed without a leading zero and b q formed once.  stag_lface_acc
// and the row-tile smoother (which stages the diagonal in place of alpha)
// evaluate these expressions, so their results agree bit for bit.
template <typename T, int DIM>
__device__ __forceinline__ T stag_diag1(T a, T b, T q) {
    return a + T(2 * DIM) * b * q;
}
template <typename T, int DIM, int C, class Own>
__device__ __forceinline__ T stag_l1_f32(Own own, T diag, T bq) {
    constexpr int ex = (C == 0), ey = (C == 1), ez = (C == 2);
    const T own_ = own(ex, ey, ez) + own(-ex, -ey, -ez);
    T o2 = T(0);
    bool first = true;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        if (d == C) continue;
        const int dx_ = (d == 0), dy_ = (d == 1), dz_ = (d == 2);
        const T pr = own(dx_, dy_, dz_) + own(-dx_, -dy_, -dz_);
        o2 = first ? pr : o2 + pr;
        first = false;
    }
    return own(0, 0, 0) * diag - (own_ + o2) * bq;
}

// (alpha_scale*alpha - L) phi on the face of component C at cell P, and the
// diagonal coefficient: the stencils of stag_applyop_2d/_3d
// (stag_applyop.f90:212-1075) and the 'fac' of stag_mg_update
// (stag_mg_solver.f90:1764-2458).
//
// The velocity values come through two accessors, own(dx,dy,dz) for
// component C and oth(d,dx,dy,dz) for component d != C, both relative to P,
// and alpha of the face through alp(); the other coefficients are read from
// global memory.  Every smoother, residual and
// operator kernel evaluates this one expression, so a value computed from
// shared-memory planes equals the one computed from global memory bit for
// bit.
template <typename T, int DIM, int VISC, int C, class CellT, class Own, class Oth, class Alp>
__device__ __forceinline__ T stag_lface_acc(const StagOp<T>& A, const CellT& P, Own own, Oth oth, Alp alp,
                                            T& diag) {
    constexpr int ex = (C == 0), ey = (C == 1), ez = (C == 2);
    const i64 f = P.id(0, 0, 0);
    const i64 fmc = P.id(-ex, -ey, -ez);
    const T ph = own(0, 0, 0);
    const T a = A.alpha_scale * alp();
    const T q = A.q;
    if constexpr (VISC < 0) {
        const T bp = ld(A.beta, f), bm = ld(A.beta, fmc);
        T kp, km;
        if constexpr (VISC == -1) {
            kp = bp; km = bm;
        } else if constexpr (VISC == -2) {
            kp = T(2) * bp; km = T(2) * bm;
        } else {
            kp = T(4.0 / 3.0) * bp + ld(A.gamma, f);
            km = T(4.0 / 3.0) * bm + ld(A.gamma, fmc);
        }
        T s = kp + km;
        T nb = own(ex, ey, ez) * kp + own(-ex, -ey, -ez) * km;
        T cross = T(0);
        T tp = T(0), tm = T(0);
        if constexpr (VISC == -3) {
            tp = -T(2.0 / 3.0) * bp + ld(A.gamma, f);
            tm = -T(2.0 / 3.0) * bm + ld(A.gamma, fmc);
        }
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            if (d == C) continue;
            const int dx_ = (d == 0), dy_ = (d == 1), dz_ = (d == 2);
            const i64 fpd = P.id(dx_, dy_, dz_);
            const T* E = A.bed[edge_of<DIM>(C, d)];
            const T elo = ld(E, f), ehi = ld(E, fpd);
            s += elo + ehi;
            nb += own(dx_, dy_, dz_) * ehi + own(-dx_, -dy_, -dz_) * elo;
            if constexpr (VISC != -1) {
                cross += oth(d, dx_, dy_, dz_) * (ehi + tp) - oth(d, 0, 0, 0) * (elo + tp) -
                         oth(d, dx_ - ex, dy_ - ey, dz_ - ez) * (ehi + tm) + oth(d, -ex, -ey, -ez) * (elo + tm);
            }
        }
        diag = a + s * q;
        return ph * diag - (nb + cross) * q;
    } else {
        const T b = A.beta0_set ? A.beta0 : ld(A.beta, 0);
        const T own_ = own(ex, ey, ez) + own(-ex, -ey, -ez);
        T oth_ = T(0), cross = T(0);
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            if (d == C) continue;
            const int dx_ = (d == 0), dy_ = (d == 1), dz_ = (d == 2);
            oth_ += own(dx_, dy_, dz_) + own(-dx_, -dy_, -dz_);
            if constexpr (VISC != 1) {
                cross += oth(d, dx_, dy_, dz_) - oth(d, 0, 0, 0) - oth(d, dx_ - ex, dy_ - ey, dz_ - ez) +
                         oth(d, -ex, -ey, -ez);
            }
        }
        if constexpr (VISC == 1) {
            diag = stag_diag1<T, DIM>(a, b, q);
            // FP32 (the multigrid of the mixed-precision solve): stag_l1_f32
            if constexpr (sizeof(T) == 4) return stag_l1_f32<T, DIM, C>(own, diag, b * q);
            return ph * diag - (own_ + oth_) * b * q;
        } else if constexpr (VISC == 2) {
            diag = a + T(2 * DIM + 2) * b * q;
            return ph * diag - (T(2) * own_ + oth_ + cross) * b * q;
        } else {
            const T cg = ld(A.gamma, 0);
            diag = a + ((T(8.0 / 3.0) + T(2 * (DIM - 1))) * b + T(2) * cg) * q;
            return ph * diag - (own_ * (T(4.0 / 3.0) * b + cg) + oth_ * b + cross * (T(1.0 / 3.0) * b + cg)) * q;
        }
    }
}

// the operator on global-memory velocity arrays
template <typename T, int DIM, int VISC, int C, class CellT>
__device__ __forceinline__ T stag_lface(const StagOp<T>& A, const T* const* phi, const CellT& P, T& diag) {
    const T* pc = phi[C];
    return stag_lface_acc<T, DIM, VISC, C>(
        A, P, [&](int a, int b, int c) { return ld(pc, P.id(a, b, c)); },
        [&](int d, int a, int b, int c) { return ld(phi[d], P.id(a, b, c)); },
        [&]() { return ld(A.alpha[C], P.id(0, 0, 0)); }, diag);
}

template <typename T, int DIM, int VISC, class CellT>
__device__ __forceinline__ T stag_lface_c(int c, const StagOp<T>& A, const T* const* phi, const CellT& P, T& diag) {
    if (c == 0) return stag_lface<T, DIM, VISC, 0>(A, phi, P, diag);
    if (DIM == 3 && c == 2) return stag_lface<T, DIM, VISC, (DIM == 3 ? 2 : 1)>(A, phi, P, diag);
    return stag_lface<T, DIM, VISC, 1>(A, phi, P, diag);
}

__device__ __forceinline__ bool cellf_of_thread(const Grid& g, CellF& P) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.n[0] || j >= g.n[1]) return false;
    P.set(g, i, j, blockIdx.z);
    return true;
}

__device__ __forceinline__ bool cell_of_thread(const Grid& g, Cell& P) {
    P.nx = g.n[0]; P.ny = g.n[1]; P.nz = g.n[2];
    P.i = blockIdx.x * blockDim.x + threadIdx.x;
    P.j = blockIdx.y * blockDim.y + threadIdx.y;
    P.k = blockIdx.z;
    return P.i < P.nx && P.j < P.ny;
}

// ---------------------------------------------------------------------
// staggered operator kernels
// ---------------------------------------------------------------------

// out[c] = L phi  (mode 0), rhs[c] - L phi (mode 1, residual)
template <typename T, int DIM, int VISC>
__global__ void __launch_bounds__(256) k_stag_apply(Grid g, StagOp<T> A, const T* __restrict__ p0,
                                                    const T* __restrict__ p1, const T* __restrict__ p2,
                                                    T* o0, T* o1, T* o2, const T* r0, const T* r1, const T* r2,
                                                    int mode) {
    CellF P;
    if (!cellf_of_thread(g, P)) return;
    const T* phi[3] = {p0, p1, p2};
    T* out[3] = {o0, o1, o2};
    const T* rhs[3] = {r0, r1, r2};
    const i64 f = P.id(0, 0, 0);
#pragma unroll
    for (int c = 0; c < DIM; c++) {
        T dg;
        T L = stag_lface_c<T, DIM, VISC>(c, A, phi, P, dg);
        out[c][f] = mode ? ld(rhs[c], f) - L : L;
    }
}

// One colour of the 2*dim-colour Gauss-Seidel smoother, fused: the
// applyop(colour) of stag_applyop_level and the stag_mg_update(colour)
// (stag_mg_solver.f90:360-396).  Faces of component C with parity
// (i+j+k)%2 == par are updated.  Valid when every extent is even (no face
// of the colour then neighbours another face of the same colour).
// Thread x-index runs over half the row.
template <typename T, int DIM, int VISC, int C>
__global__ void __launch_bounds__(256) k_stag_gs(Grid g, StagOp<T> A, T* p0, T* p1, T* p2,
                                                 const T* __restrict__ r, int par, T omega) {
    const int ih = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (j >= g.n[1]) return;
    const int i = 2 * ih + ((j + k + par) & 1);
    if (i >= g.n[0]) return;
    CellF P;
    P.set(g, i, j, k);
    const T* phi[3] = {p0, p1, p2};
    T* pc = (C == 0) ? p0 : (C == 1 ? p1 : p2);
    const i64 f = P.id(0, 0, 0);
    T dg;
    const T L = stag_lface<T, DIM, VISC, C>(A, phi, P, dg);
    pc[f] = pc[f] + sm_quot(omega * (ld(r, f) - L), dg);
}

// Two-pass colour smoother for levels with an odd extent or the Jacobi
// smoother (colour 0): pass 1 stores L phi and the diagonal for the colour.
template <typename T, int DIM, int VISC>
__global__ void __launch_bounds__(256) k_stag_color_apply(Grid g, StagOp<T> A, const T* p0, const T* p1,
                                                          const T* p2, T* L0, T* L1, T* L2, T* D0, T* D1, T* D2,
                                                          int color) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    const T* phi[3] = {p0, p1, p2};
    T* Lo[3] = {L0, L1, L2};
    T* Do[3] = {D0, D1, D2};
    const i64 f = P.id(0, 0, 0);
    const int par = (P.i + P.j + P.k) & 1;
#pragma unroll
    for (int c = 0; c < DIM; c++) {
        if (color != 0 && ((color - 1) / 2 != c || par != ((color + 1) & 1))) continue;
        T dg;
        Lo[c][f] = stag_lface_c<T, DIM, VISC>(c, A, phi, P, dg);
        Do[c][f] = dg;
    }
}

template <typename T, int DIM>
__global__ void __launch_bounds__(256) k_stag_color_update(Grid g, T* p0, T* p1, T* p2, const T* r0, const T* r1,
                                                           const T* r2, const T* L0, const T* L1, const T* L2,
                                                           const T* D0, const T* D1, const T* D2, int color,
                                                           T omega) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    T* ph[3] = {p0, p1, p2};
    const T* rh[3] = {r0, r1, r2};
    const T* Lo[3] = {L0, L1, L2};
    const T* Do[3] = {D0, D1, D2};
    const i64 f = P.id(0, 0, 0);
    const int par = (P.i + P.j + P.k) & 1;
#pragma unroll
    for (int c = 0; c < DIM; c++) {
        if (color != 0 && ((color - 1) / 2 != c || par != ((color + 1) & 1))) continue;
        ph[c][f] = ph[c][f] + sm_quot(omega * (rh[c][f] - Lo[c][f]), Do[c][f]);
    }
}

// stag_restriction (stag_mg_solver.f90:1028-1170): 6-point (2D) / 12-point
// (3D) full stencil, or the 2/4-point 'simple' stencil, of one component.
// The fine values come through at(o, pa, pb): the fine face at offset o
// along the component and pa, pb along the two other directions from the
// fine cell 2Q of coarse cell Q.
template <typename T, int DIM, class At>
__device__ __forceinline__ T stag_restrict_expr(int simple, At at) {
    if constexpr (DIM == 2) {
        if (simple) return T(0.5) * (at(0, 0, 0) + at(0, 1, 0));
        return T(0.25) * (at(0, 0, 0) + at(0, 1, 0)) +
               T(0.125) * (at(1, 0, 0) + at(1, 1, 0) + at(-1, 0, 0) + at(-1, 1, 0));
    } else {
        if (simple) return T(0.25) * (at(0, 0, 0) + at(0, 1, 0) + at(0, 0, 1) + at(0, 1, 1));
        return T(0.125) * (at(0, 0, 0) + at(0, 1, 0) + at(0, 0, 1) + at(0, 1, 1)) +
               T(0.0625) * (at(1, 0, 0) + at(1, 1, 0) + at(1, 0, 1) + at(1, 1, 1)) +
               T(0.0625) * (at(-1, 0, 0) + at(-1, 1, 0) + at(-1, 0, 1) + at(-1, 1, 1));
    }
}

// stag_prolongation (stag_mg_solver.f90:1419-1628) of one component at a
// fine face: coarse values through at(o, pa, pb) relative to the parent
// cell; even = the face lies on a coarse face; oa, ob = the side of the
// neighbouring coarse row in the two other directions
template <typename T, int DIM, class At>
__device__ __forceinline__ T stag_prolong_expr(bool even, int oa, int ob, At at) {
    if constexpr (DIM == 2) {
        if (even) return T(0.75) * at(0, 0, 0) + T(0.25) * at(0, oa, 0);
        return T(0.375) * at(0, 0, 0) + T(0.125) * at(0, oa, 0) + T(0.375) * at(1, 0, 0) + T(0.125) * at(1, oa, 0);
    } else {
        if (even)
            return T(9.0 / 16.0) * at(0, 0, 0) + T(3.0 / 16.0) * at(0, oa, 0) + T(3.0 / 16.0) * at(0, 0, ob) +
                   T(1.0 / 16.0) * at(0, oa, ob);
        return T(9.0 / 32.0) * at(0, 0, 0) + T(3.0 / 32.0) * at(0, oa, 0) + T(3.0 / 32.0) * at(0, 0, ob) +
               T(1.0 / 32.0) * at(0, oa, ob) + T(9.0 / 32.0) * at(1, 0, 0) + T(3.0 / 32.0) * at(1, oa, 0) +
               T(3.0 / 32.0) * at(1, 0, ob) + T(1.0 / 32.0) * at(1, oa, ob);
    }
}

// fine face (or coarse cell) of component c at the offset (o, pa, pb) in
// component-relative directions: the linear index through Cell X
template <int DIM>
__device__ __forceinline__ i64 comp_off_id(const Cell& X, int c, int o, int pa, int pb) {
    const int a = (c == 0) ? 1 : 0;
    const int b = (c == 2) ? 1 : 2;
    int off[3] = {0, 0, 0};
    off[c] += o;
    off[a] += pa;
    if (DIM == 3) off[b] += pb;
    return X.id(off[0], off[1], off[2]);
}

// Thread per coarse cell, all components.
template <typename T, int DIM>
__global__ void __launch_bounds__(256) k_stag_restrict(Grid gf, Grid gc, const T* f0, const T* f1, const T* f2,
                                                       T* c0, T* c1, T* c2, int simple) {
    Cell Q;
    if (!cell_of_thread(gc, Q)) return;
    Cell F;
    F.nx = gf.n[0]; F.ny = gf.n[1]; F.nz = gf.n[2];
    F.i = 2 * Q.i; F.j = 2 * Q.j; F.k = (DIM == 3) ? 2 * Q.k : 0;
    const T* fi[3] = {f0, f1, f2};
    T* co[3] = {c0, c1, c2};
    const i64 qc = Q.id(0, 0, 0);
#pragma unroll
    for (int c = 0; c < DIM; c++) {
        const T* Fp = fi[c];
        co[c][qc] = stag_restrict_expr<T, DIM>(
            simple, [&](int o, int pa, int pb) { return ld(Fp, comp_off_id<DIM>(F, c, o, pa, pb)); });
    }
}

// two consecutive elements (an x-pair of fine cells), one vector access
template <typename T>
struct Pair2;
template <>
struct Pair2<float> {
    typedef float2 V;
};
template <>
struct Pair2<double> {
    typedef double2 V;
};

// fine += P coarse.  Thread per coarse cell: per component the 18 coarse
// faces that its 2x2x2 fine children read (offsets 0, 1 along the
// component, -1..1 across it) are loaded once, and the children's x-pairs
// are read and written as one vector each (vec: every fine array is aligned
// to two elements; else two scalar accesses).  Every fine value is the
// stag_prolong_expr of the per-fine-cell form.
template <typename T, int DIM>
__global__ void __launch_bounds__(256) k_stag_prolong(Grid gf, Grid gc, T* f0, T* f1, T* f2, const T* c0,
                                                      const T* c1, const T* c2, int vec) {
    typedef typename Pair2<T>::V V2;
    CellF H;
    if ((int)blockIdx.z >= gc.n[2] || !cellf_of_thread(gc, H)) return;
    const i64 nxf = gf.n[0], nxyf = (i64)gf.n[0] * gf.n[1];
    const i64 fb = 2 * (i64)H.i + nxf * 2 * H.j + (DIM == 3 ? nxyf * 2 * H.k : 0);
    T* fo[3] = {f0, f1, f2};
    const T* ci[3] = {c0, c1, c2};
#pragma unroll
    for (int c = 0; c < DIM; c++) {
        const int a = (c == 0) ? 1 : 0;
        const int b = (c == 2) ? 1 : 2;
        T cv[2][3][3];
#pragma unroll
        for (int o = 0; o < 2; o++)
#pragma unroll
            for (int pa = -1; pa <= 1; pa++)
#pragma unroll
                for (int pb = -1; pb <= 1; pb++) {
                    if (DIM == 2 && pb != 0) continue;
                    int off[3] = {0, 0, 0};
                    off[c] += o;
                    off[a] += pa;
                    if (DIM == 3) off[b] += pb;
                    cv[o][pa + 1][pb + 1] = ld(ci[c], H.id(off[0], off[1], off[2]));
                }
#pragma unroll
        for (int pz = 0; pz < (DIM == 3 ? 2 : 1); pz++)
#pragma unroll
            for (int py = 0; py < 2; py++) {
                T* row = fo[c] + fb + py * nxf + pz * nxyf;
                T out[2];
                if (vec) {
                    const V2 v = *reinterpret_cast<const V2*>(row);
                    out[0] = v.x;
                    out[1] = v.y;
                } else {
                    out[0] = row[0];
                    out[1] = row[1];
                }
#pragma unroll
                for (int px = 0; px < 2; px++) {
                    const int I[3] = {px, py, pz};  // parities of the fine indices
                    const int oa = I[a] ? 1 : -1;
                    const int ob = (DIM == 3) ? (I[b] ? 1 : -1) : 0;
                    out[px] = out[px] + stag_prolong_expr<T, DIM>(
                                            I[c] == 0, oa, ob,
                                            [&](int o, int qa, int qb) { return cv[o][qa + 1][qb + 1]; });
                }
                if (vec) {
                    V2 v;
                    v.x = out[0];
                    v.y = out[1];
                    *reinterpret_cast<V2*>(row) = v;
                } else {
                    row[0] = out[0];
                    row[1] = out[1];
                }
            }
    }
}

// k_stag_prolong's vector flag for the fine arrays f[0..dim)
template <typename T>
inline int pair_aligned(int dim, T* const* f) {
    for (int c = 0; c < dim; c++)
        if ((uintptr_t)f[c] % (2 * sizeof(T))) return 0;
    return 1;
}

// cc_restriction (stag_mg_solver.f90:919-963): average of 2^dim children
template <typename T, int DIM>
__global__ void __launch_bounds__(256) k_cc_average(Grid gf, Grid gc, const T* F, T* Cc) {
    Cell Q;
    if (!cell_of_thread(gc, Q)) return;
    Cell P;
    P.nx = gf.n[0]; P.ny = gf.n[1]; P.nz = gf.n[2];
    P.i = 2 * Q.i; P.j = 2 * Q.j; P.k = (DIM == 3) ? 2 * Q.k : 0;
    T v;
    if constexpr (DIM == 2) {
        v = T(0.25) * (ld(F, P.id(0, 0, 0)) + ld(F, P.id(1, 0, 0)) + ld(F, P.id(0, 1, 0)) + ld(F, P.id(1, 1, 0)));
    } else {
        v = T(0.125) * (ld(F, P.id(0, 0, 0)) + ld(F, P.id(1, 0, 0)) + ld(F, P.id(0, 1, 0)) + ld(F, P.id(1, 1, 0)) +
                        ld(F, P.id(0, 0, 1)) + ld(F, P.id(1, 0, 1)) + ld(F, P.id(0, 1, 1)) + ld(F, P.id(1, 1, 1)));
    }
    Cc[Q.id(0, 0, 0)] = v;
}

// nodal_restriction (2D injection) / edge_restriction (3D 2-point),
// stag_mg_solver.f90:1173-1362
template <typename T, int DIM>
__global__ void __launch_bounds__(256) k_edge_coarsen(Grid gf, Grid gc, const T* e0, const T* e1, const T* e2,
                                                      T* c0, T* c1, T* c2) {
    Cell Q;
    if (!cell_of_thread(gc, Q)) return;
    Cell P;
    P.nx = gf.n[0]; P.ny = gf.n[1]; P.nz = gf.n[2];
    P.i = 2 * Q.i; P.j = 2 * Q.j; P.k = (DIM == 3) ? 2 * Q.k : 0;
    const i64 q = Q.id(0, 0, 0);
    if constexpr (DIM == 2) {
        c0[q] = ld(e0, P.id(0, 0, 0));
    } else {
        c0[q] = T(0.5) * (ld(e0, P.id(0, 0, 0)) + ld(e0, P.id(0, 0, 1)));
        c1[q] = T(0.5) * (ld(e1, P.id(0, 0, 0)) + ld(e1, P.id(0, 1, 0)));
        c2[q] = T(0.5) * (ld(e2, P.id(0, 0, 0)) + ld(e2, P.id(1, 0, 0)));
    }
}

// ---------------------------------------------------------------------
// cell-centred pressure multigrid (FBoxLib ml_cc_solve as used by
// macproject.f90:294-298, semantics of PreconditionerNotes.tex:484-575)
// ---------------------------------------------------------------------
template <typename T>
struct CCOp {
    const T* a[3];  // face coefficient (alphainv), low side of each cell
    T q;            // 1/dx^2 of the level
};

// D a G phi at cell P and its diagonal; phi through the accessor
// ph(dx,dy,dz) relative to P (global memory or shared-memory planes, one
// expression for both)
template <typename T, int DIM, class CellT, class Acc>
__device__ __forceinline__ T cc_lap_acc(const CCOp<T>& A, const CellT& P, Acc ph, T& diag) {
    const i64 f = P.id(0, 0, 0);
    const T pc = ph(0, 0, 0);
    T s = T(0), dg = T(0);
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        const int dx_ = (d == 0), dy_ = (d == 1), dz_ = (d == 2);
        const i64 fp = P.id(dx_, dy_, dz_);
        const T ahi = ld(A.a[d], fp), alo = ld(A.a[d], f);
        s += ahi * (ph(dx_, dy_, dz_) - pc) - alo * (pc - ph(-dx_, -dy_, -dz_));
        dg += ahi + alo;
    }
    diag = -dg * A.q;
    return s * A.q;
}

template <typename T, int DIM, class CellT>
__device__ __forceinline__ T cc_lap(const CCOp<T>& A, const T* phi, const CellT& P, T& diag) {
    return cc_lap_acc<T, DIM>(A, P, [&](int a, int b, int c) { return ld(phi, P.id(a, b, c)); }, diag);
}

// red-black Gauss-Seidel, one colour, fused; thread per cell of the colour
template <typename T, int DIM>
__global__ void __launch_bounds__(256) k_cc_gsrb(Grid g, CCOp<T> A, T* phi, const T* __restrict__ rhs, int par) {
    const int ih = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (j >= g.n[1]) return;
    const int i = 2 * ih + ((j + k + par) & 1);
    if (i >= g.n[0]) return;
    CellF P;
    P.set(g, i, j, k);
    T dg;
    const T L = cc_lap<T, DIM>(A, phi, P, dg);
    const i64 f = P.id(0, 0, 0);
    phi[f] = phi[f] + sm_quot(ld(rhs, f) - L, dg);
}

// two-pass colour for odd extents: store the correction, then add it
template <typename T, int DIM>
__global__ void __launch_bounds__(256) k_cc_color_corr(Grid g, CCOp<T> A, const T* phi, const T* rhs, T* corr,
                                                       int par) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    if (((P.i + P.j + P.k) & 1) != par) return;
    T dg;
    const T L = cc_lap<T, DIM>(A, phi, P, dg);
    const i64 f = P.id(0, 0, 0);
    corr[f] = sm_quot(ld(rhs, f) - L, dg);
}

template <typename T>
__global__ void __launch_bounds__(256) k_cc_color_add(Grid g, T* phi, const T* corr, int par) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    if (((P.i + P.j + P.k) & 1) != par) return;
    const i64 f = P.id(0, 0, 0);
    phi[f] = phi[f] + corr[f];
}

// residual on the 2^dim children of coarse cell (qi, qj, qk), averaged:
// the coarse rhs (residual + restriction in one pass; every fine cell once).
// phi_at / rhs_at read the fine arrays by linear index.
template <typename T, int DIM, class PhiAt, class RhsAt>
__device__ __forceinline__ T cc_resid_avg(const CCOp<T>& A, const Grid& gf, int qi, int qj, int qk, PhiAt phi_at,
                                          RhsAt rhs_at) {
    Cell P;
    P.nx = gf.n[0]; P.ny = gf.n[1]; P.nz = gf.n[2];
    T acc = T(0);
    const int kz = (DIM == 3) ? 2 : 1;
#pragma unroll
    for (int dk = 0; dk < kz; dk++)
#pragma unroll
        for (int dj = 0; dj < 2; dj++)
#pragma unroll
            for (int di = 0; di < 2; di++) {
                P.i = 2 * qi + di; P.j = 2 * qj + dj; P.k = (DIM == 3) ? 2 * qk + dk : 0;
                T dg;
                const T L = cc_lap_acc<T, DIM>(A, P, [&](int a, int b, int c) { return phi_at(P.id(a, b, c)); }, dg);
                acc += rhs_at(P.id(0, 0, 0)) - L;
            }
    return acc * (DIM == 3 ? T(0.125) : T(0.25));
}

template <typename T, int DIM>
__global__ void __launch_bounds__(256) k_cc_resid_restrict(Grid gf, Grid gc, CCOp<T> A, const T* phi, const T* rhs,
                                                           T* crhs) {
    Cell Q;
    if (!cell_of_thread(gc, Q)) return;
    crhs[Q.id(0, 0, 0)] = cc_resid_avg<T, DIM>(
        A, gf, Q.i, Q.j, Q.k, [&](i64 i) { return ld(phi, i); }, [&](i64 i) { return ld(rhs, i); });
}

// phi += coarse phi of the parent cell.  Thread per coarse cell, its fine
// children written as x-pairs.
template <typename T, int DIM>
__global__ void __launch_bounds__(256) k_cc_prolong(Grid gf, Grid gc, T* phi, const T* cphi) {
    typedef typename Pair2<T>::V V2;
    Cell Q;
    if ((int)blockIdx.z >= gc.n[2] || !cell_of_thread(gc, Q)) return;
    const T cv = ld(cphi, Q.id(0, 0, 0));
    const i64 nxf = gf.n[0], nxyf = (i64)gf.n[0] * gf.n[1];
    const i64 fb = 2 * (i64)Q.i + nxf * 2 * Q.j + (DIM == 3 ? nxyf * 2 * Q.k : 0);
#pragma unroll
    for (int pz = 0; pz < (DIM == 3 ? 2 : 1); pz++)
#pragma unroll
        for (int py = 0; py < 2; py++) {
            V2* row = reinterpret_cast<V2*>(phi + fb + py * nxf + pz * nxyf);
            V2 v = *row;
            v.x = v.x + cv;
            v.y = v.y + cv;
            *row = v;
        }
}

template <typename T, int DIM>
__global__ void __launch_bounds__(256) k_cc_resid(Grid g, CCOp<T> A, const T* phi, const T* rhs, T* res) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    T dg;
    const i64 f = P.id(0, 0, 0);
    res[f] = ld(rhs, f) - cc_lap<T, DIM>(A, phi, P, dg);
}

}  // namespace fhd
