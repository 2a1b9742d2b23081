// fhd_solver.cu -- staggered multigrid, pressure multigrid, the
// preconditioner, the saddle-point operator and GMRES, driven from the host
// on one CUDA stream; plus the device-pointer C ABI.
//
// Follows staggered_grid/src_gmres of LowMachFHD: gmres.f90,
// apply_matrix.f90, apply_precon.f90, stag_mg_solver.f90, macproject.f90.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <map>

#include "fhd_solver.cuh"
#include "fhd_coarse.cuh"
#include "fhd_rbx.cuh"

namespace fhd {

static thread_local std::string g_last_error;
void set_last_error(const std::string& s) { g_last_error = s; }

static std::mutex g_pinned_mu;
static std::vector<double*> g_pinned_free;

double* pinned_scalars_acquire() {
    {
        std::lock_guard<std::mutex> lk(g_pinned_mu);
        if (!g_pinned_free.empty()) {
            double* p = g_pinned_free.back();
            g_pinned_free.pop_back();
            return p;
        }
    }
    double* p = nullptr;
    if (cudaMallocHost((void**)&p, sizeof(double) * 256) != cudaSuccess) return nullptr;
    return p;
}

void pinned_scalars_release(double* p) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(g_pinned_mu);
    g_pinned_free.push_back(p);
}

int nlevs_mg(const Grid& g, int minwidth) {
    // compute_nlevs_mg (stag_mg_layout.f90:179-222), one box
    int nl = -1;
    for (int d = 0; d < g.dim; d++) {
        int t = g.n[d], r = 1;
        while (t % 2 == 0 && t / minwidth != 1) {
            t /= 2;
            r++;
        }
        nl = (nl < 0) ? r : (r < nl ? r : nl);
    }
    return nl;
}

static inline int post(fhd_ctx* ctx) {
    ctx->launches++;
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) {
        set_last_error(std::string("kernel launch: ") + cudaGetErrorString(e));
        return FHD_ERR_CUDA;
    }
    return 0;
}

#define FHD_POST(ctx)                 \
    do {                              \
        int rc_ = post(ctx);          \
        if (rc_) return rc_;          \
    } while (0)

template <typename T>
static Multigrid<T>& mg_of(fhd_ctx* ctx);
template <>
Multigrid<double>& mg_of<double>(fhd_ctx* ctx) { return ctx->mg64; }
template <>
Multigrid<float>& mg_of<float>(fhd_ctx* ctx) { return ctx->mg32; }

// ---------------------------------------------------------------------
// hierarchy construction (stag_mg_layout_build / mgt_macproj_precon_build)
// ---------------------------------------------------------------------
// levels of the multi-box staggered hierarchy and whether its bottom is the
// fancy nested solve (stag_mg_layout.f90:21-107, stag_mg_solver.f90:97-101,
// 447): boxes of max_grid_size cells where that is below the domain extent
static void stag_box_layout(fhd_ctx* ctx, int ns_domain) {
    ctx->stag_nl_box = 0;
    ctx->stag_fancy = false;
    bool any = false, multi = true;
    int nb[3] = {ctx->n[0], ctx->n[1], ctx->n[2]};
    for (int d = 0; d < ctx->dim; d++) {
        const int m = ctx->mgs[d];
        if (m <= 0 || m >= ctx->n[d]) {
            multi = false;
            continue;
        }
        nb[d] = m;
        any = true;
    }
    if (!any) return;
    const Grid gb = make_grid(ctx->dim, nb, ctx->dx);
    const int nlb = nlevs_mg(gb, ctx->p.stag_mg_minwidth);
    if (nlb >= ns_domain) return;
    ctx->stag_nl_box = nlb;
    ctx->stag_fancy = ctx->p.stag_mg_bottom_solver == 4 && multi;
}

template <typename T>
static int build_mg(fhd_ctx* ctx, Multigrid<T>& M) {
    const int dim = ctx->dim;
    const int nE = dim == 2 ? 1 : 3;
    Arena& A = ctx->arena;
    int ns = nlevs_mg(ctx->g0, ctx->p.stag_mg_minwidth);
    stag_box_layout(ctx, ns);
    // several boxes without the fancy bottom: the hierarchy of the boxes
    if (ctx->stag_nl_box > 0 && !ctx->stag_fancy) ns = ctx->stag_nl_box;
    M.s.resize(ns);
    for (int l = 0; l < ns; l++) {
        StagLevel<T>& L = M.s[l];
        L.g = (l == 0) ? ctx->g0 : coarsen(M.s[l - 1].g);
        const i64 nc = L.g.nc;
        for (int c = 0; c < dim; c++) {
            if (l > 0) {
                L.alpha[c] = A.alloc<T>(nc);
                L.phi[c] = A.alloc<T>(nc);
                L.rhs[c] = A.alloc<T>(nc);
                if (!L.alpha[c] || !L.phi[c] || !L.rhs[c]) return FHD_ERR_OOM;
            }
            L.tmp[c] = A.alloc<T>(nc);
            if (!L.tmp[c]) return FHD_ERR_OOM;
            if (!all_even(L.g) || ctx->p.stag_mg_smoother == 0) {
                L.diag[c] = A.alloc<T>(nc);
                if (!L.diag[c]) return FHD_ERR_OOM;
            }
        }
        if (l > 0 || !std::is_same<T, double>::value) {
            L.own_beta = A.alloc<T>(nc);
            L.own_gamma = A.alloc<T>(nc);
            if (!L.own_beta || !L.own_gamma) return FHD_ERR_OOM;
            for (int e = 0; e < nE; e++) {
                L.own_bed[e] = A.alloc<T>(nc);
                if (!L.own_bed[e]) return FHD_ERR_OOM;
            }
            L.beta = L.own_beta;
            L.gamma = L.own_gamma;
            for (int e = 0; e < nE; e++) L.bed[e] = L.own_bed[e];
        }
        if (l == 0 && !std::is_same<T, double>::value) {
            for (int c = 0; c < dim; c++) {
                L.own_alpha0[c] = A.alloc<T>(nc);
                if (!L.own_alpha0[c]) return FHD_ERR_OOM;
                L.alpha[c] = L.own_alpha0[c];
            }
        }
        // the levels the row-tile smoother can take (rbx_geom: FP32, 3D,
        // visc_type 1, x extent 64 to 256)
        if (!std::is_same<T, double>::value && dim == 3 && ctx->visc == 1 && L.g.n[0] >= 64 &&
            L.g.n[0] <= RBX_MAXNX)
            for (int c = 0; c < 3; c++) {
                L.rbx_diag[c] = A.alloc<T>(nc);
                if (!L.rbx_diag[c]) return FHD_ERR_OOM;
            }
    }
    const int ncl = nlevs_mg(ctx->g0, ctx->p.mg_minwidth);
    M.c.resize(ncl);
    for (int l = 0; l < ncl; l++) {
        CCLevel<T>& C = M.c[l];
        C.g = (l == 0) ? ctx->g0 : coarsen(M.c[l - 1].g);
        const i64 nc = C.g.nc;
        for (int c = 0; c < dim; c++) {
            C.a[c] = A.alloc<T>(nc);
            if (!C.a[c]) return FHD_ERR_OOM;
            if (ctx->p.visc_schur_approx != 0) {
                C.amu[c] = A.alloc<T>(nc);
                if (!C.amu[c]) return FHD_ERR_OOM;
            }
        }
        C.phi = A.alloc<T>(nc);
        C.rhs = A.alloc<T>(nc);
        C.tmp = A.alloc<T>(nc);
        if (!C.phi || !C.rhs || !C.tmp) return FHD_ERR_OOM;
    }
    const i64 nc0 = ctx->g0.nc;
    for (int c = 0; c < dim; c++) {
        M.x_u[c] = A.alloc<T>(nc0);
        M.b_u[c] = A.alloc<T>(nc0);
        if (!M.x_u[c] || !M.b_u[c]) return FHD_ERR_OOM;
    }
    M.mac_rhs = A.alloc<T>(nc0);
    if (!M.mac_rhs) return FHD_ERR_OOM;
    if (ctx->p.visc_schur_approx != 0) {
        for (int c = 0; c < dim; c++)
            if (!(M.bf_g[c] = A.alloc<T>(nc0))) return FHD_ERR_OOM;
        if (!(M.bf_phi = A.alloc<T>(nc0))) return FHD_ERR_OOM;
    }
    return 0;
}

// coefficient hierarchy for the current operator (stag_mg_solver.f90:
// 200-230; alphainv of apply_precon.f90:73-76 coarsened for the pressure
// multigrid as face averages)
// zero the wall faces of a face vector of level grid g (no-op without walls)
template <typename T>
static int zero_walls(fhd_ctx* ctx, const Grid& g, T* u0, T* u1, T* u2) {
    if (!ctx->has_walls) return 0;
    int rc = 0;
    with_dim(ctx->dim, [&](auto D) {
        constexpr int DIM = decltype(D)::value;
        k_zero_walls<T, DIM><<<cell_grid(g), cell_block(), 0, ctx->stream>>>(g, ctx->walls, u0, u1, u2);
        rc |= post(ctx);
    });
    return rc;
}

// the wall smoother is two-pass on every staggered level: the diagonal
// arrays that only odd-extent levels have otherwise
template <typename T>
static int wall_diag(fhd_ctx* ctx) {
    for (auto& L : mg_of<T>(ctx).s)
        for (int c = 0; c < ctx->dim; c++)
            if (!L.diag[c]) {
                L.diag[c] = ctx->arena.alloc<T>(L.g.nc);
                if (!L.diag[c]) return FHD_ERR_OOM;
            }
    return 0;
}

// the visc_type 1 diagonal of one component (stag_diag1, the expression of
// stag_lface_acc) for the row-tile smoother; beta is constant (beta[0])
template <typename T, int DIM>
__global__ void __launch_bounds__(256) k_stag_diag1(i64 n, T* out, const T* alpha, T alpha_scale, const T* beta,
                                                    T q) {
    const T b = beta[0];
    for (i64 f = blockIdx.x * (i64)blockDim.x + threadIdx.x; f < n; f += (i64)gridDim.x * blockDim.x)
        out[f] = stag_diag1<T, DIM>(alpha_scale * alpha[f], b, q);
}

template <typename T>
static int prepare_T(fhd_ctx* ctx) {
    Multigrid<T>& M = mg_of<T>(ctx);
    const int dim = ctx->dim;
    const int nE = dim == 2 ? 1 : 3;
    const i64 nc0 = ctx->g0.nc;
    cudaStream_t st = ctx->stream;
    StagLevel<T>& L0 = M.s[0];
    if (std::is_same<T, double>::value) {
        for (int c = 0; c < dim; c++) L0.alpha[c] = (T*)ctx->alpha_fc[c];
        L0.alpha_scale = (T)ctx->theta;
        L0.beta = (const T*)ctx->beta;
        L0.gamma = (const T*)ctx->gamma;
        for (int e = 0; e < nE; e++) L0.bed[e] = (const T*)ctx->beta_ed[e];
    } else {
        const int nb = flat_blocks(nc0);
        for (int c = 0; c < dim; c++) {
            k_copy_conv<T, double><<<nb, 256, 0, st>>>(nc0, L0.own_alpha0[c], ctx->alpha_fc[c], ctx->theta);
            FHD_POST(ctx);
        }
        L0.alpha_scale = T(1);
        k_copy_conv<T, double><<<nb, 256, 0, st>>>(nc0, L0.own_beta, ctx->beta, 1.0);
        FHD_POST(ctx);
        k_copy_conv<T, double><<<nb, 256, 0, st>>>(nc0, L0.own_gamma, ctx->gamma, 1.0);
        FHD_POST(ctx);
        for (int e = 0; e < nE; e++) {
            k_copy_conv<T, double><<<nb, 256, 0, st>>>(nc0, L0.own_bed[e], ctx->beta_ed[e], 1.0);
            FHD_POST(ctx);
        }
    }
    for (size_t l = 1; l < M.s.size(); l++) {
        StagLevel<T>& F = M.s[l - 1];
        StagLevel<T>& C = M.s[l];
        int rc = 0;
        with_dim(dim, [&](auto D) {
            constexpr int DIM = decltype(D)::value;
            k_cc_average<T, DIM><<<cell_grid(C.g), cell_block(), 0, st>>>(F.g, C.g, F.beta, C.own_beta);
            rc |= post(ctx);
            k_cc_average<T, DIM><<<cell_grid(C.g), cell_block(), 0, st>>>(F.g, C.g, F.gamma, C.own_gamma);
            rc |= post(ctx);
            k_edge_coarsen<T, DIM><<<cell_grid(C.g), cell_block(), 0, st>>>(
                F.g, C.g, F.bed[0], F.bed[1], F.bed[2], C.own_bed[0], C.own_bed[1], C.own_bed[2]);
            rc |= post(ctx);
        });
        if (rc) return rc;
        if (l == 1 && F.alpha_scale != T(1)) {
            // level 0 alpha carries theta_alpha through alpha_scale: form
            // theta*alpha in the level-1 buffer first, then coarsen
            // in place is not possible; scale while restricting instead
            const int nb = flat_blocks(F.g.nc);
            for (int c = 0; c < dim; c++) {
                k_copy_conv<T, T><<<nb, 256, 0, st>>>(F.g.nc, F.tmp[c], F.alpha[c], (double)F.alpha_scale);
                FHD_POST(ctx);
            }
            with_dim(dim, [&](auto D) {
                constexpr int DIM = decltype(D)::value;
                k_stag_restrict<T, DIM><<<cell_grid(C.g), cell_block(), 0, st>>>(
                    F.g, C.g, F.tmp[0], F.tmp[1], F.tmp[2], C.alpha[0], C.alpha[1], C.alpha[2], 1);
                rc |= post(ctx);
            });
        } else {
            with_dim(dim, [&](auto D) {
                constexpr int DIM = decltype(D)::value;
                k_stag_restrict<T, DIM><<<cell_grid(C.g), cell_block(), 0, st>>>(
                    F.g, C.g, F.alpha[0], F.alpha[1], F.alpha[2], C.alpha[0], C.alpha[1], C.alpha[2], 1);
                rc |= post(ctx);
            });
        }
        if (rc) return rc;
        C.alpha_scale = T(1);
    }
    for (StagLevel<T>& L : M.s) {
        if (!L.rbx_diag[0]) continue;
        const StagOp<T> A = L.op();
        const int nb = flat_blocks(L.g.nc);
        for (int c = 0; c < 3; c++) {
            k_stag_diag1<T, 3><<<nb, 256, 0, st>>>(L.g.nc, L.rbx_diag[c], L.alpha[c], L.alpha_scale, L.beta, A.q);
            FHD_POST(ctx);
        }
    }
    // pressure multigrid coefficients: alphainv on the finest level
    {
        const int nb = flat_blocks(nc0);
        for (int c = 0; c < dim; c++) {
            k_recip<T><<<nb, 256, 0, st>>>(nc0, M.c[0].a[c], ctx->alpha_fc[c]);
            FHD_POST(ctx);
        }
        for (size_t l = 1; l < M.c.size(); l++) {
            CCLevel<T>& F = M.c[l - 1];
            CCLevel<T>& C = M.c[l];
            int rc = 0;
            with_dim(dim, [&](auto D) {
                constexpr int DIM = decltype(D)::value;
                k_stag_restrict<T, DIM><<<cell_grid(C.g), cell_block(), 0, st>>>(
                    F.g, C.g, F.a[0], F.a[1], F.a[2], C.a[0], C.a[1], C.a[2], 1);
                rc |= post(ctx);
            });
            if (rc) return rc;
        }
        // walls: no flux through a wall face (with the periodic index wrap
        // of the pressure kernels the high wall face is face 0 as well)
        for (size_t l = 0; l < M.c.size(); l++)
            if (int rc = zero_walls<T>(ctx, M.c[l].g, M.c[l].a[0], M.c[l].a[1], M.c[l].a[2])) return rc;
    }
    // the BFBt pressure multigrid: mu^-1 = 1/diag(viscous operator)
    // (apply_precon.f90:589), coarsened as alpha^-1 is
    if (ctx->p.visc_schur_approx != 0) {
        int rc = 0;
        CCLevel<T>& C0 = M.c[0];
        with_dim(dim, [&](auto D) {
            constexpr int DIM = decltype(D)::value;
            k_inv_diag_lap<T, DIM><<<cell_grid(C0.g), cell_block(), 0, st>>>(
                C0.g, ctx->visc, ctx->beta, ctx->beta_ed[0], ctx->beta_ed[1], ctx->beta_ed[2], C0.amu[0], C0.amu[1],
                C0.amu[2]);
            rc |= post(ctx);
            for (size_t l = 1; l < M.c.size(); l++) {
                CCLevel<T>& F = M.c[l - 1];
                CCLevel<T>& C = M.c[l];
                k_stag_restrict<T, DIM><<<cell_grid(C.g), cell_block(), 0, st>>>(
                    F.g, C.g, F.amu[0], F.amu[1], F.amu[2], C.amu[0], C.amu[1], C.amu[2], 1);
                rc |= post(ctx);
            }
        });
        if (rc) return rc;
    }
    return 0;
}

template <typename T>
static int tune_levels(fhd_ctx* ctx);

int prepare(fhd_ctx* ctx, const double* const alpha_fc[], const double* beta, const double* const beta_ed[],
            const double* gamma, double theta) {
    const int dim = ctx->dim;
    for (int c = 0; c < 3; c++) ctx->alpha_fc[c] = c < dim ? alpha_fc[c] : nullptr;
    ctx->beta = beta;
    ctx->gamma = gamma;
    for (int e = 0; e < 3; e++) ctx->beta_ed[e] = e < (dim == 2 ? 1 : 3) ? beta_ed[e] : nullptr;
    ctx->theta = theta;
    if (ctx->prec == FHD_PREC_MIXED) {
        int rc = prepare_T<float>(ctx);
        return rc ? rc : tune_levels<float>(ctx);
    }
    int rc = prepare_T<double>(ctx);
    return rc ? rc : tune_levels<double>(ctx);
}

// ---------------------------------------------------------------------
// staggered multigrid V-cycle (stag_mg_solver.f90:323-808)
// ---------------------------------------------------------------------
// algorithmic bytes of one fused colour sweep of component c: the whole
// component array is read (the colour and its neighbours), the colour's
// rhs and alpha read and the colour written; variable coefficients add the
// cell and edge viscosities, cross terms the other components
template <typename T>
static double gs_sweep_bytes(fhd_ctx* ctx, const StagLevel<T>& L) {
    const double nc = (double)L.g.nc, s = (double)sizeof(T);
    const int dim = ctx->dim, v = ctx->visc;
    double words = nc + 1.5 * nc;
    if (v < 0) words += nc + (dim - 1) * nc;
    if (v == 2 || v == -2 || v == 3 || v == -3) words += (dim - 1) * nc;
    if (v == -3) words += nc;
    return words * s;
}

static cudaEvent_t prof_event(fhd_ctx* ctx) {
    if (ctx->prof_used >= ctx->prof_ev.size()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        ctx->prof_ev.push_back(e);
    }
    return ctx->prof_ev[ctx->prof_used++];
}

// one profiling timestamp on stream st.  Inside a graph capture the record
// becomes an event-record node of the graph; its handle is kept (in capture
// order) so that every replay can point it at a fresh event.
static void prof_mark(fhd_ctx* ctx, cudaStream_t st) {
    if (!ctx->capturing) {
        cudaEventRecord(prof_event(ctx), st);
        return;
    }
    // an external record is a graph node (a plain record inside a capture
    // only orders streams and leaves no node)
    cudaEventRecordWithFlags(prof_event(ctx), st, cudaEventRecordExternal);
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    if (cudaStreamGetCaptureInfo(st, &cs, nullptr, nullptr, &deps, &nd) == cudaSuccess && nd == 1)
        ctx->cap_nodes.push_back(deps[0]);
    else
        ctx->cap_fail = true;
}

// colour launches over the cells of one colour with thread block blk
inline dim3 half_grid_for(const Grid& g, dim3 blk) {
    return dim3(((g.n[0] + 1) / 2 + blk.x - 1) / blk.x, (g.n[1] + blk.y - 1) / blk.y, g.n[2]);
}

template <typename T>
static int stag_smooth(fhd_ctx* ctx, StagLevel<T>& L, int color, dim3 blk = cell_block()) {
    cudaStream_t st = ctx->stream;
    const dim3 hg = half_grid_for(L.g, blk);
    const T omega = (T)ctx->p.stag_mg_omega;
    const StagOp<T> A = L.op();
    int rc = 0;
    if (color != 0 && all_even(L.g)) {
        const bool timed = ctx->prof && L.g.nc == ctx->g0.nc;
        if (timed) {
            prof_mark(ctx, st);
            ctx->prof_bytes += gs_sweep_bytes(ctx, L);
            ctx->prof_launches++;
        }
        const int c = (color - 1) / 2;
        const int par = (color + 1) & 1;
        with_dim_visc(ctx->dim, ctx->visc, [&](auto D, auto V) {
            constexpr int DIM = decltype(D)::value, VISC = decltype(V)::value;
            if (c == 0)
                k_stag_gs<T, DIM, VISC, 0><<<hg, blk, 0, st>>>(L.g, A, L.phi[0], L.phi[1], L.phi[2], L.rhs[0], par,
                                                               omega);
            else if (c == 1)
                k_stag_gs<T, DIM, VISC, 1><<<hg, blk, 0, st>>>(L.g, A, L.phi[0], L.phi[1], L.phi[2], L.rhs[1], par,
                                                               omega);
            else
                k_stag_gs<T, DIM, VISC, (DIM == 3 ? 2 : 1)><<<hg, blk, 0, st>>>(
                    L.g, A, L.phi[0], L.phi[1], L.phi[2], L.rhs[DIM == 3 ? 2 : 1], par, omega);
            rc |= post(ctx);
        });
        if (timed) prof_mark(ctx, st);
        return rc;
    }
    with_dim_visc(ctx->dim, ctx->visc, [&](auto D, auto V) {
        constexpr int DIM = decltype(D)::value, VISC = decltype(V)::value;
        k_stag_color_apply<T, DIM, VISC><<<cell_grid(L.g), cell_block(), 0, st>>>(
            L.g, A, L.phi[0], L.phi[1], L.phi[2], L.tmp[0], L.tmp[1], L.tmp[2], L.diag[0], L.diag[1], L.diag[2],
            color);
        rc |= post(ctx);
        k_stag_color_update<T, DIM><<<cell_grid(L.g), cell_block(), 0, st>>>(
            L.g, L.phi[0], L.phi[1], L.phi[2], L.rhs[0], L.rhs[1], L.rhs[2], L.tmp[0], L.tmp[1], L.tmp[2],
            L.diag[0], L.diag[1], L.diag[2], color, omega);
        rc |= post(ctx);
    });
    return rc;
}

// algorithmic bytes of one fused smooth launch (all colours of the
// components it covers): src, rhs, alpha read and dst written per component,
// plus the variable viscosities and, for coupled operators, the other
// components
template <typename T>
static double rb_smooth_bytes(fhd_ctx* ctx, const StagLevel<T>& L) {
    const double nc = (double)L.g.nc, s = (double)sizeof(T);
    const int v = ctx->visc;
    double words = 4.0 * nc;
    if (v < 0) words += nc + 2.0 * nc;
    if (v == -3) words += nc;
    if (v != 1 && v != -1) words += 2.0 * nc;
    return words * s * ((v == 1 || v == -1) ? 3.0 : 1.0);
}

// dynamic shared memory above the 48 KB default: raise each kernel's limit
// (keyed by device and kernel address) to the largest size launched so far
// (full_carveout: also ask for the whole unified L1 / shared-memory array as
// shared memory, so that two large CTAs fit on one SM)
template <class K>
static int rb_allow_smem(K kernel, size_t bytes, bool full_carveout = false) {
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, size_t> done;
    if (bytes <= 48 * 1024) return 0;
    int dev = 0;
    FHD_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    size_t& d = done[std::make_pair(dev, (const void*)kernel)];
    if (bytes <= d) return 0;
    FHD_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    if (full_carveout)
        FHD_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                          (int)cudaSharedmemCarveoutMaxShared));
    d = bytes;
    return 0;
}

// one full smooth a -> b of every component (3D, even extents)
template <typename T>
static int stag_rb_smooth(fhd_ctx* ctx, StagLevel<T>& L, const RBGeom& G, T* const a[3], T* const b[3]) {
    const StagOp<T> A = L.op();
    const T omega = (T)ctx->p.stag_mg_omega;
    const size_t smem = rb_smem<T>(G, 2);
    cudaStream_t st = ctx->stream;
    const dim3 blk(32, G.TY + 1);
    int rc = 0;
    RBArgs<T> R;
    for (int c = 0; c < 3; c++) {
        R.src[c] = a[c];
        R.dst[c] = b[c];
        R.rhs[c] = L.rhs[c];
        R.oth[c] = nullptr;
    }
    const bool timed = ctx->prof && L.g.nc == ctx->g0.nc;
    with_visc3(ctx->visc, [&](auto V) {
        constexpr int VISC = decltype(V)::value;
        if constexpr (VISC == 1 || VISC == -1) {
            if (timed) {
                prof_mark(ctx, st);
                ctx->prof_bytes += rb_smooth_bytes(ctx, L);
                ctx->prof_launches++;
            }
            rc |= rb_allow_smem(k_stag_rb<T, VISC, -1>, smem);
            k_stag_rb<T, VISC, -1><<<dim3(G.tiles_x * G.tiles_y, G.chunks, 3), blk, smem, st>>>(L.g, G, A, R, omega);
            rc |= post(ctx);
            if (timed) prof_mark(ctx, st);
        } else {
            const dim3 grd(G.tiles_x * G.tiles_y, G.chunks, 1);
            for (int c = 0; c < 3; c++) {
                // components before c already hold this smooth's values
                for (int d = 0; d < 3; d++) R.oth[d] = d < c ? b[d] : a[d];
                if (timed) {
                    prof_mark(ctx, st);
                    ctx->prof_bytes += rb_smooth_bytes(ctx, L);
                    ctx->prof_launches++;
                }
                rc |= rb_allow_smem(k_stag_rb<T, VISC, 0>, smem);
                rc |= rb_allow_smem(k_stag_rb<T, VISC, 1>, smem);
                rc |= rb_allow_smem(k_stag_rb<T, VISC, 2>, smem);
                if (c == 0) k_stag_rb<T, VISC, 0><<<grd, blk, smem, st>>>(L.g, G, A, R, omega);
                else if (c == 1) k_stag_rb<T, VISC, 1><<<grd, blk, smem, st>>>(L.g, G, A, R, omega);
                else k_stag_rb<T, VISC, 2><<<grd, blk, smem, st>>>(L.g, G, A, R, omega);
                rc |= post(ctx);
                if (timed) prof_mark(ctx, st);
            }
        }
    });
    return rc;
}

// one full smooth a -> b of every component with the row-tile smoother
// (FP32, visc_type 1)
static int stag_rbx_smooth(fhd_ctx* ctx, StagLevel<float>& L, const RBXGeom& G, float* const a[3],
                           float* const b[3]) {
    RBXArgs R;
    for (int c = 0; c < 3; c++) {
        R.src[c] = a[c];
        R.dst[c] = b[c];
        R.rhs[c] = L.rhs[c];
        R.diag[c] = L.rbx_diag[c];
    }
    if (!R.diag[0]) return FHD_ERR_UNSUPPORTED;
    R.err = ctx->dev_err;
    const bool timed = ctx->prof && L.g.nc == ctx->g0.nc;
    if (timed) {
        prof_mark(ctx, ctx->stream);
        ctx->prof_bytes += rb_smooth_bytes(ctx, L);
        ctx->prof_launches++;
    }
    const dim3 grd(G.chunks, 1, 1);
    if (G.ahead == 1) {
        if (int rc = rb_allow_smem(k_stag_rbx<1>, G.smem, true)) return rc;
        k_stag_rbx<1><<<grd, RBX_BLOCK, G.smem, ctx->stream>>>(L.g, G, L.op(), R, (float)ctx->p.stag_mg_omega);
    } else if (G.threads == 512) {
        if (int rc = rb_allow_smem(k_stag_rbx<RBX_AHEAD, 512>, G.smem)) return rc;
        k_stag_rbx<RBX_AHEAD, 512><<<grd, 512 + 32, G.smem, ctx->stream>>>(L.g, G, L.op(), R,
                                                                          (float)ctx->p.stag_mg_omega);
    } else {
        if (int rc = rb_allow_smem(k_stag_rbx<RBX_AHEAD>, G.smem)) return rc;
        k_stag_rbx<RBX_AHEAD><<<grd, RBX_BLOCK, G.smem, ctx->stream>>>(L.g, G, L.op(), R,
                                                                      (float)ctx->p.stag_mg_omega);
    }
    int rc = post(ctx);
    if (timed) prof_mark(ctx, ctx->stream);
    return rc;
}

template <typename T>
static bool stag_aligned(const StagLevel<T>& L, int dim) {
    bool aligned = true;
    for (int c = 0; c < dim; c++)
        aligned = aligned && rb_aligned(L.phi[c]) && rb_aligned(L.tmp[c]) && rb_aligned(L.rhs[c]) &&
                  rb_aligned(L.alpha[c]) && (!L.rbx_diag[c] || rb_aligned(L.rbx_diag[c]));
    return aligned;
}

// count smooths of a level as its tuned plan says: pairs of fused smooths
// phi -> tmp -> phi (kinds 1, 2), colour launches for the rest
template <typename T>
static int stag_smooths_planned(fhd_ctx* ctx, StagLevel<T>& L, const SmoothPlan& P, int count) {
    int m0 = 0;
    T* a[3] = {L.phi[0], L.phi[1], L.phi[2]};
    T* b[3] = {L.tmp[0], L.tmp[1], L.tmp[2]};
    if constexpr (std::is_same<T, float>::value) {
        if (P.kind == 2)
            for (; m0 + 2 <= count; m0 += 2) {
                int rc = stag_rbx_smooth(ctx, L, P.rbx, a, b);
                if (!rc) rc = stag_rbx_smooth(ctx, L, P.rbx, b, a);
                if (rc) return rc;
            }
    }
    if (P.kind == 1)
        for (; m0 + 2 <= count; m0 += 2) {
            int rc = stag_rb_smooth(ctx, L, P.rb, a, b);
            if (!rc) rc = stag_rb_smooth(ctx, L, P.rb, b, a);
            if (rc) return rc;
        }
    const dim3 blk(P.kind == 0 ? P.bx : 32, P.kind == 0 ? P.by : 8, 1);
    for (int m = m0; m < count; m++)
        for (int color = 1; color <= 2 * ctx->dim; color++) {
            int rc = stag_smooth(ctx, L, color, blk);
            if (rc) return rc;
        }
    return 0;
}

template <typename T>
static int stag_smooths(fhd_ctx* ctx, StagLevel<T>& L, int count) {
    const int dim = ctx->dim;
    if (ctx->has_walls) {
        // the colours of the reference's smoother, each as Lphi and the
        // diagonal of its faces, then the update (the wall faces stay zero)
        const StagOp<T> A = L.op();
        const T omega = (T)ctx->p.stag_mg_omega;
        int rc = 0;
        for (int m = 0; m < count && !rc; m++)
            for (int color = 1; color <= 2 * dim && !rc; color++)
                with_dim_wall_visc(dim, ctx->visc, [&](auto D, auto V) {
                    constexpr int DIM = decltype(D)::value, VISC = decltype(V)::value;
                    k_stag_color_apply_w<T, DIM, VISC><<<cell_grid(L.g), cell_block(), 0, ctx->stream>>>(
                        L.g, ctx->walls, A, L.phi[0], L.phi[1], L.phi[2], L.rhs[0], L.rhs[1], L.rhs[2], L.tmp[0],
                        L.tmp[1], L.tmp[2], L.diag[0], L.diag[1], L.diag[2], color);
                    rc |= post(ctx);
                    k_stag_color_update<T, DIM><<<cell_grid(L.g), cell_block(), 0, ctx->stream>>>(
                        L.g, L.phi[0], L.phi[1], L.phi[2], L.rhs[0], L.rhs[1], L.rhs[2], L.tmp[0], L.tmp[1],
                        L.tmp[2], L.diag[0], L.diag[1], L.diag[2], color, omega);
                    rc |= post(ctx);
                });
        return rc;
    }
    int m0 = 0;
    RBGeom G;
    const bool aligned = stag_aligned(L, dim);
    if (L.plan.kind >= 0 && ctx->fused_mode != 0 && ctx->p.stag_mg_smoother != 0 && aligned && all_even(L.g))
        return stag_smooths_planned(ctx, L, L.plan, count);
    if constexpr (std::is_same<T, float>::value) {
        RBXGeom X;
        if (ctx->p.stag_mg_smoother != 0 && ctx->visc == 1 && count >= 2 && aligned && !rb_use(L.g) &&
            ctx->fused_mode != 0 && rbx_geom(L.g, ctx->sms, (size_t)ctx->smem_optin, X)) {
            float* a[3] = {L.phi[0], L.phi[1], L.phi[2]};
            float* b[3] = {L.tmp[0], L.tmp[1], L.tmp[2]};
            for (; m0 + 2 <= count; m0 += 2) {
                int rc = stag_rbx_smooth(ctx, L, X, a, b);
                if (rc) return rc;
                rc = stag_rbx_smooth(ctx, L, X, b, a);
                if (rc) return rc;
            }
        }
    }
    if (ctx->p.stag_mg_smoother != 0 && count - m0 >= 2 && aligned && rb_use(L.g) &&
        rb_geom(L.g, 3, (int)sizeof(T), G)) {
        // pairs of fused smooths phi -> tmp -> phi
        T* a[3] = {L.phi[0], L.phi[1], L.phi[2]};
        T* b[3] = {L.tmp[0], L.tmp[1], L.tmp[2]};
        for (; m0 + 2 <= count; m0 += 2) {
            int rc = stag_rb_smooth(ctx, L, G, a, b);
            if (rc) return rc;
            rc = stag_rb_smooth(ctx, L, G, b, a);
            if (rc) return rc;
        }
    }
    for (int m = m0; m < count; m++) {
        if (ctx->p.stag_mg_smoother == 0) {
            int rc = stag_smooth(ctx, L, 0);
            if (rc) return rc;
        } else {
            for (int color = 1; color <= 2 * dim; color++) {
                int rc = stag_smooth(ctx, L, color);
                if (rc) return rc;
            }
        }
    }
    return 0;
}

template <typename T>
static int stag_residual(fhd_ctx* ctx, StagLevel<T>& L) {
    int rc = 0;
    const StagOp<T> A = L.op();
    if (ctx->has_walls) {
        with_dim_wall_visc(ctx->dim, ctx->visc, [&](auto D, auto V) {
            constexpr int DIM = decltype(D)::value, VISC = decltype(V)::value;
            k_stag_apply_w<T, DIM, VISC><<<cell_grid(L.g), cell_block(), 0, ctx->stream>>>(
                L.g, ctx->walls, A, L.phi[0], L.phi[1], L.phi[2], L.tmp[0], L.tmp[1], L.tmp[2], L.rhs[0], L.rhs[1],
                L.rhs[2], 1);
            rc |= post(ctx);
        });
        return rc;
    }
    with_dim_visc(ctx->dim, ctx->visc, [&](auto D, auto V) {
        constexpr int DIM = decltype(D)::value, VISC = decltype(V)::value;
        k_stag_apply<T, DIM, VISC><<<cell_grid(L.g), cell_block(), 0, ctx->stream>>>(
            L.g, A, L.phi[0], L.phi[1], L.phi[2], L.tmp[0], L.tmp[1], L.tmp[2], L.rhs[0], L.rhs[1], L.rhs[2], 1);
        rc |= post(ctx);
    });
    return rc;
}

// shared memory one coarse kernel may take: the device's opt-in limit less a
// margin for the L1 that caches the coefficients
static size_t coarse_smem_cap() {
    int dev = 0, optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 0;
    const size_t cap = 200 * 1024;
    return (size_t)optin < cap ? (size_t)optin : cap;
}

// first level of a hierarchy of n levels that the single-CTA coarse kernel
// takes over (every level from it to the bottom fits the shared-memory
// cap; level l needs bytes(l)); n when none does or the mode is off
template <class F>
static int coarse_first(fhd_ctx* ctx, int n, F bytes) {
    if (ctx->coarse_mode == 0) return n;
    const size_t cap = coarse_smem_cap();
    size_t tot = 0;
    int lc = n;
    for (int l = n - 1; l >= 0 && n - l <= CS_MAXL; l--) {
        tot += bytes(l);
        if (tot > cap) break;
        lc = l;
    }
    return lc;
}

template <typename T>
static int stag_coarse_first(fhd_ctx* ctx, Multigrid<T>& M) {
    const int dim = ctx->dim;
    // the single-CTA coarse kernel knows no walls: every level by launches
    if (ctx->has_walls) return (int)M.s.size();
    return coarse_first(ctx, (int)M.s.size(),
                        [&](int l) { return (size_t)(3 * dim) * (size_t)M.s[l].g.nc * sizeof(T); });
}

template <typename T>
static int cc_coarse_first(fhd_ctx* ctx, Multigrid<T>& M) {
    return coarse_first(ctx, (int)M.c.size(), [&](int l) { return (size_t)3 * (size_t)M.c[l].g.nc * sizeof(T); });
}

// levels lc..bottom of the staggered V-cycle in one CTA: phi of level lc in
// global memory is the input (lc == 0) or zero, and holds the result
template <typename T>
static int stag_coarse(fhd_ctx* ctx, Multigrid<T>& M, int lc) {
    const int nl = (int)M.s.size();
    const int dim = ctx->dim;
    StagCoarseArgs<T> a;
    memset(&a, 0, sizeof a);
    a.nlev = nl - lc;
    a.load_phi = lc == 0;
    a.n_down = ctx->p.stag_mg_nsmooths_down;
    a.n_up = ctx->p.stag_mg_nsmooths_up;
    a.n_bottom = ctx->p.stag_mg_nsmooths_bottom;
    a.jacobi = ctx->p.stag_mg_smoother == 0;
    a.omega = (T)ctx->p.stag_mg_omega;
    for (int c = 0; c < dim; c++) {
        a.phi[c] = M.s[lc].phi[c];
        a.rhs[c] = M.s[lc].rhs[c];
    }
    size_t off = 0;
    for (int m = 0; m < a.nlev; m++) {
        const StagLevel<T>& L = M.s[lc + m];
        a.g[m] = L.g;
        a.A[m] = L.op();
        a.off[m] = (int)off;
        off += (size_t)(3 * dim) * (size_t)L.g.nc;
    }
    const size_t smem = off * sizeof(T);
    int rc = 0;
    with_dim_visc(dim, ctx->visc, [&](auto D, auto V) {
        constexpr int DIM = decltype(D)::value, VISC = decltype(V)::value;
        rc |= rb_allow_smem(k_stag_coarse<T, DIM, VISC>, smem);
        if (rc) return;
        k_stag_coarse<T, DIM, VISC><<<1, CS_THREADS, smem, ctx->stream>>>(a);
        rc |= post(ctx);
    });
    return rc;
}

template <typename T>
static int stag_vcycle(fhd_ctx* ctx, Multigrid<T>& M) {
    const int nl = (int)M.s.size();
    const int dim = ctx->dim;
    cudaStream_t st = ctx->stream;
    // levels from lc down run in the coarse kernel, which zeroes their phi
    const int lc = stag_coarse_first(ctx, M);
    const int lt = lc < nl - 1 ? lc : nl - 1;  // last level of the per-level descent
    for (int l = 1; l < lc; l++)
        for (int c = 0; c < dim; c++) FHD_CUDA_TRY(cudaMemsetAsync(M.s[l].phi[c], 0, sizeof(T) * M.s[l].g.nc, st));
    for (int l = 0; l < lt; l++) {
        StagLevel<T>& L = M.s[l];
        StagLevel<T>& C = M.s[l + 1];
        int rc = stag_smooths(ctx, L, ctx->p.stag_mg_nsmooths_down);
        if (rc) return rc;
        rc = stag_residual(ctx, L);
        if (rc) return rc;
        with_dim(dim, [&](auto D) {
            constexpr int DIM = decltype(D)::value;
            k_stag_restrict<T, DIM><<<cell_grid(C.g), cell_block(), 0, st>>>(L.g, C.g, L.tmp[0], L.tmp[1], L.tmp[2],
                                                                           C.rhs[0], C.rhs[1], C.rhs[2], 0);
            rc |= post(ctx);
        });
        // the restricted residual is zero on the coarse wall faces
        if (!rc) rc = zero_walls<T>(ctx, C.g, C.rhs[0], C.rhs[1], C.rhs[2]);
        if (rc) return rc;
    }
    int rc = lc < nl ? stag_coarse(ctx, M, lc) : stag_smooths(ctx, M.s[nl - 1], ctx->p.stag_mg_nsmooths_bottom);
    if (rc) return rc;
    for (int l = lt - 1; l >= 0; l--) {
        StagLevel<T>& L = M.s[l];
        StagLevel<T>& C = M.s[l + 1];
        if (ctx->has_walls) {
            with_dim(dim, [&](auto D) {
                constexpr int DIM = decltype(D)::value;
                k_stag_prolong_w<T, DIM><<<cell_grid(L.g), cell_block(), 0, st>>>(
                    L.g, C.g, ctx->walls, L.phi[0], L.phi[1], L.phi[2], C.phi[0], C.phi[1], C.phi[2]);
                rc |= post(ctx);
            });
        } else {
            with_dim(dim, [&](auto D) {
                constexpr int DIM = decltype(D)::value;
                k_stag_prolong<T, DIM><<<cell_grid(C.g), cell_block(), 0, st>>>(
                    L.g, C.g, L.phi[0], L.phi[1], L.phi[2], C.phi[0], C.phi[1], C.phi[2], pair_aligned(dim, L.phi));
                rc |= post(ctx);
            });
        }
        if (rc) return rc;
        rc = stag_smooths(ctx, L, ctx->p.stag_mg_nsmooths_up);
        if (rc) return rc;
    }
    return 0;
}

template <typename T>
static int maxabs_resid(fhd_ctx* ctx, StagLevel<T>& L, double* out);

// max |a| per array, via sum-free reduction into host
template <typename T>
__global__ void __launch_bounds__(RED_THREADS) k_maxabs(i64 n, const T* a, RedSlot rs) {
    double s = 0.0;
    for (i64 f = blockIdx.x * (i64)blockDim.x + threadIdx.x; f < n; f += (i64)gridDim.x * blockDim.x)
        s = fmax(s, fabs((double)a[f]));
    // max-combine: reuse the sum tree on a monotone transform is not exact,
    // so reduce the maxima explicitly
    __shared__ double sh[RED_THREADS];
    __shared__ bool last;
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        rs.partials[blockIdx.x] = sh[0];
        __threadfence();
        last = (atomicAdd(rs.counter, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int b = 0; b < (int)gridDim.x; b++) m = fmax(m, ((volatile double*)rs.partials)[b]);
        *rs.out = m;
        *rs.counter = 0u;
    }
}

template <typename T>
static int stag_mg_run(fhd_ctx* ctx, Multigrid<T>& M);

// one V-cycle of the multi-box hierarchy whose bottom, level lb, is the
// fancy nested stag_mg_solver (stag_mg_solver.f90:447-555): levels lb ..
// nl-1 of M form the re-boxed bottom problem's own hierarchy; its V-cycle
// count is restored afterwards, as the reference restores vcycle_counter
template <typename T>
static int stag_vcycle_fancy(fhd_ctx* ctx, Multigrid<T>& M, int lb) {
    const int nl = (int)M.s.size();
    const int dim = ctx->dim;
    cudaStream_t st = ctx->stream;
    for (int l = 1; l < nl; l++)
        for (int c = 0; c < dim; c++) FHD_CUDA_TRY(cudaMemsetAsync(M.s[l].phi[c], 0, sizeof(T) * M.s[l].g.nc, st));
    for (int l = 0; l < lb; l++) {
        StagLevel<T>& L = M.s[l];
        StagLevel<T>& C = M.s[l + 1];
        int rc = stag_smooths(ctx, L, ctx->p.stag_mg_nsmooths_down);
        if (!rc) rc = stag_residual(ctx, L);
        if (rc) return rc;
        with_dim(dim, [&](auto D) {
            constexpr int DIM = decltype(D)::value;
            k_stag_restrict<T, DIM><<<cell_grid(C.g), cell_block(), 0, st>>>(L.g, C.g, L.tmp[0], L.tmp[1], L.tmp[2],
                                                                           C.rhs[0], C.rhs[1], C.rhs[2], 0);
            rc |= post(ctx);
        });
        if (rc) return rc;
    }
    Multigrid<T> B;  // a view of levels lb .. nl-1 (the levels' arrays are shared)
    B.s.assign(M.s.begin() + lb, M.s.end());
    const int vsaved = ctx->vcycles;
    int rc = stag_mg_run(ctx, B);
    ctx->vcycles = vsaved;
    if (rc) return rc;
    for (int l = lb - 1; l >= 0; l--) {
        StagLevel<T>& L = M.s[l];
        StagLevel<T>& C = M.s[l + 1];
        with_dim(dim, [&](auto D) {
            constexpr int DIM = decltype(D)::value;
            k_stag_prolong<T, DIM><<<cell_grid(C.g), cell_block(), 0, st>>>(L.g, C.g, L.phi[0], L.phi[1], L.phi[2],
                                                                          C.phi[0], C.phi[1], C.phi[2],
                                                                          pair_aligned(dim, L.phi));
            rc |= post(ctx);
        });
        if (rc) return rc;
        rc = stag_smooths(ctx, L, ctx->p.stag_mg_nsmooths_up);
        if (rc) return rc;
    }
    return 0;
}

// stag_mg_solver (stag_mg_solver.f90:37-863) on level-0 phi/rhs of M
template <typename T>
static int stag_mg_run(fhd_ctx* ctx, Multigrid<T>& M) {
    const int dim = ctx->dim;
    const int maxv = ctx->p.stag_mg_max_vcycles;
    StagLevel<T>& L0 = M.s[0];
    const i64 nc = L0.g.nc;
    if (int rc = zero_walls<T>(ctx, L0.g, L0.phi[0], L0.phi[1], L0.phi[2])) return rc;
    double resid0[3] = {0, 0, 0};
    if (maxv > 1) {
        int rc = stag_residual(ctx, L0);
        if (rc) return rc;
        for (int c = 0; c < dim; c++) {
            k_maxabs<T><<<flat_blocks(nc), RED_THREADS, 0, ctx->stream>>>(nc, L0.tmp[c], slot(ctx, S_MG + c));
            FHD_POST(ctx);
        }
        rc = sync_scalars(ctx, S_MG, dim);
        if (rc) return rc;
        bool allzero = true, anyzero = false;
        double rmax = 0;
        for (int c = 0; c < dim; c++) {
            resid0[c] = ctx->hscal[S_MG + c];
            allzero = allzero && resid0[c] == 0.0;
            anyzero = anyzero || resid0[c] == 0.0;
            rmax = fmax(rmax, resid0[c]);
        }
        if (allzero) return 0;
        if (anyzero)
            for (int c = 0; c < dim; c++) resid0[c] = rmax;
    }
    // the fancy bottom changes the cycle only when its nested solve may take
    // more than one V-cycle: with one, the nested cycle smooths the shared
    // level before and after it exactly as an intermediate level is smoothed
    const bool nested = ctx->stag_fancy && maxv > 1 && M.s.size() == mg_of<T>(ctx).s.size() &&
                        ctx->stag_nl_box > 1 && ctx->stag_nl_box < (int)M.s.size();
    for (int vc = 1; vc <= maxv; vc++) {
        int rc = nested ? stag_vcycle_fancy(ctx, M, ctx->stag_nl_box - 1) : stag_vcycle(ctx, M);
        if (rc) return rc;
        if (vc == maxv) break;
        rc = stag_residual(ctx, L0);
        if (rc) return rc;
        for (int c = 0; c < dim; c++) {
            k_maxabs<T><<<flat_blocks(nc), RED_THREADS, 0, ctx->stream>>>(nc, L0.tmp[c], slot(ctx, S_MG + c));
            FHD_POST(ctx);
        }
        rc = sync_scalars(ctx, S_MG, dim);
        if (rc) return rc;
        bool done = true;
        for (int c = 0; c < dim; c++) done = done && (ctx->hscal[S_MG + c] / resid0[c] < ctx->p.stag_mg_rel_tol);
        if (done) break;
    }
    ctx->vcycles += dim * maxv;
    return 0;
}

// ---------------------------------------------------------------------
// pressure multigrid (macproject.f90:34-316)
// ---------------------------------------------------------------------
template <typename T>
static int cc_smooth(fhd_ctx* ctx, CCLevel<T>& C, dim3 blk = cell_block()) {
    cudaStream_t st = ctx->stream;
    const CCOp<T> A = C.op();
    const dim3 hg = half_grid_for(C.g, blk);
    int rc = 0;
    for (int par = 0; par < 2; par++) {
        with_dim(ctx->dim, [&](auto D) {
            constexpr int DIM = decltype(D)::value;
            if (all_even(C.g)) {
                k_cc_gsrb<T, DIM><<<hg, blk, 0, st>>>(C.g, A, C.phi, C.rhs, par);
                rc |= post(ctx);
            } else {
                k_cc_color_corr<T, DIM><<<cell_grid(C.g), cell_block(), 0, st>>>(C.g, A, C.phi, C.rhs, C.tmp, par);
                rc |= post(ctx);
                k_cc_color_add<T><<<cell_grid(C.g), cell_block(), 0, st>>>(C.g, C.phi, C.tmp, par);
                rc |= post(ctx);
            }
        });
        if (rc) return rc;
    }
    return 0;
}

// count red-black smooths: fused pairs phi -> tmp -> phi where the level
// allows, single colour-pair smooths otherwise
// pairs of tiled fused smooths phi -> tmp -> phi with geometry G
template <typename T>
static int cc_rb_pairs(fhd_ctx* ctx, CCLevel<T>& C, const RBGeom& G, int pairs) {
    const size_t smem = rb_smem<T>(G, 1);
    if (int rc = rb_allow_smem(k_cc_rb<T>, smem)) return rc;
    const dim3 grd(G.tiles_x * G.tiles_y, G.chunks, 1), blk(32, G.TY + 1);
    for (int m = 0; m < pairs; m++) {
        k_cc_rb<T><<<grd, blk, smem, ctx->stream>>>(C.g, G, C.op(), C.phi, C.tmp, C.rhs);
        FHD_POST(ctx);
        k_cc_rb<T><<<grd, blk, smem, ctx->stream>>>(C.g, G, C.op(), C.tmp, C.phi, C.rhs);
        FHD_POST(ctx);
    }
    return 0;
}

template <typename T>
static int cc_smooths(fhd_ctx* ctx, CCLevel<T>& C, int count) {
    int m0 = 0;
    RBGeom G;
    const bool aligned = rb_aligned(C.phi) && rb_aligned(C.tmp) && rb_aligned(C.rhs);
    if (C.plan.kind >= 0 && aligned && all_even(C.g)) {
        const SmoothPlan& P = C.plan;
        if (P.kind == 1) {
            if (int rc = cc_rb_pairs(ctx, C, P.rb, count / 2)) return rc;
            m0 = count / 2 * 2;
        }
        const dim3 blk(P.kind == 0 ? P.bx : 32, P.kind == 0 ? P.by : 8, 1);
        for (int m = m0; m < count; m++)
            if (int rc = cc_smooth(ctx, C, blk)) return rc;
        return 0;
    }
    if (count >= 2 && aligned && rb_use(C.g) && rb_geom(C.g, 1, (int)sizeof(T), G)) {
        const size_t smem = rb_smem<T>(G, 1);
        if (int rc = rb_allow_smem(k_cc_rb<T>, smem)) return rc;
        const dim3 grd(G.tiles_x * G.tiles_y, G.chunks, 1), blk(32, G.TY + 1);
        for (; m0 + 2 <= count; m0 += 2) {
            k_cc_rb<T><<<grd, blk, smem, ctx->stream>>>(C.g, G, C.op(), C.phi, C.tmp, C.rhs);
            FHD_POST(ctx);
            k_cc_rb<T><<<grd, blk, smem, ctx->stream>>>(C.g, G, C.op(), C.tmp, C.phi, C.rhs);
            FHD_POST(ctx);
        }
    }
    for (int m = m0; m < count; m++) {
        int rc = cc_smooth(ctx, C);
        if (rc) return rc;
    }
    return 0;
}

// ---------------------------------------------------------------------
// smoother autotuner
// ---------------------------------------------------------------------
// For every level that smooths through launches (above the single-CTA
// coarse end), the candidate plans -- colour launches with four thread-block
// shapes, the tiled fused smooth with several tile sizes, the row-tile
// smooth with every tile height that fits -- are timed once per process,
// device and level shape with CUDA events, and the fastest is kept.  The
// timing runs on scratch unknowns and right-hand sides (zero) with the
// level's own prepared coefficients, before any capture, so a solve's data
// is never touched.  Every plan evaluates the same update expression on the
// same operands in the same colour order: the choice changes time only.

constexpr int TUNE_REPS = 3;  // timed smooth pairs per candidate (after one untimed)

static std::mutex g_tune_mu;  // held while a context tunes
static std::map<std::string, SmoothPlan> g_tune;
static std::map<std::string, int> g_tune_import;  // imported choices (candidate index) not yet used

// A plan is keyed by the level shape and by what decides the candidate
// list: the device's SM count and shared-memory limits, and the version of
// the candidate lists (bumped whenever a list, its order or a candidate's
// kernel changes), so a table from another GPU model or library version
// selects nothing.
constexpr int TUNE_CANDS_VERSION = 5;

static std::string tune_key_of(int dev, int which, int elem, int dim, int visc, const int n[3], int sms, int optin,
                               int smem_sm) {
    char b[200];
    snprintf(b, sizeof b, "v%d:%d:%c:%d:%d:%d:%dx%dx%d:%d:%d:%d", TUNE_CANDS_VERSION, dev, which ? 'c' : 's', elem, dim,
             which ? 0 : visc, n[0], n[1], n[2], sms, optin, smem_sm);
    return b;
}

static std::string tune_key(fhd_ctx* ctx, const Grid& g, int which, int elem) {
    int dev = 0;
    cudaGetDevice(&dev);
    return tune_key_of(dev, which, elem, g.dim, ctx->visc, g.n, ctx->sms, ctx->smem_optin, ctx->smem_sm);
}

static void colour_cands(std::vector<SmoothPlan>& v, const Grid& g) {
    static const int shapes[4][2] = {{32, 8}, {64, 4}, {128, 2}, {16, 16}};
    const int hx = (g.n[0] + 1) / 2;  // cells of one colour per row
    for (const auto& sh : shapes) {
        if (sh[0] > 32 && sh[0] > 2 * hx) continue;  // more than half of every block idle
        SmoothPlan p;
        p.kind = 0;
        p.bx = sh[0];
        p.by = sh[1];
        v.push_back(p);
    }
}

// tiled fused smooth: the default tile and its narrower / shorter variants
static void rb_cands(std::vector<SmoothPlan>& v, const Grid& g, int ncomp, int elem, int ncoef, int smem_optin) {
    RBGeom G0;
    if (!rb_geom(g, ncomp, elem, G0)) return;
    const int txs[3] = {G0.TX, 32, 16}, tys[3] = {G0.TY, 8, 4};
    for (int tx : txs)
        for (int ty : tys) {
            RBGeom G;
            if (!rb_geom(g, ncomp, elem, G, tx, ty)) continue;
            const size_t smem = (size_t)elem * ((size_t)RB_NPH * G.W * G.rows + (size_t)ncoef * RB_NCF * G.W * G.crows);
            if (smem > (size_t)smem_optin) continue;
            bool dup = false;
            for (const auto& q : v) dup = dup || (q.kind == 1 && q.rb.TX == G.TX && q.rb.TY == G.TY);
            if (dup) continue;
            SmoothPlan p;
            p.kind = 1;
            p.rb = G;
            v.push_back(p);
        }
}

template <typename T>
static std::vector<SmoothPlan> stag_cands(fhd_ctx* ctx, const StagLevel<T>& L) {
    std::vector<SmoothPlan> v;
    colour_cands(v, L.g);
    rb_cands(v, L.g, 3, (int)sizeof(T), 2, ctx->smem_optin);
    if (std::is_same<T, float>::value && ctx->visc == 1)
        for (int form = 0; form < 3; form++)  // deep ring; short ring, two CTAs per SM; deep ring, 512 threads
            for (int ty = 4; ty <= 32; ty *= 2) {
                RBXGeom X;
                const int ahead = form == 1 ? 1 : RBX_AHEAD, nt = form == 2 ? 512 : RBX_THREADS;
                if (!rbx_geom(L.g, ctx->sms, (size_t)ctx->smem_optin, X, ty, ahead, (size_t)ctx->smem_sm, nt))
                    continue;
                SmoothPlan p;
                p.kind = 2;
                p.rbx = X;
                v.push_back(p);
            }
    return v;
}

template <typename T>
static std::vector<SmoothPlan> cc_cands(fhd_ctx* ctx, const CCLevel<T>& C) {
    std::vector<SmoothPlan> v;
    colour_cands(v, C.g);
    rb_cands(v, C.g, 1, (int)sizeof(T), 1, ctx->smem_optin);
    return v;
}

// one untimed smooth pair, then TUNE_REPS timed pairs; us = time of a pair
template <class F>
static int time_pairs(fhd_ctx* ctx, cudaEvent_t e0, cudaEvent_t e1, F&& pair, float& us) {
    if (int rc = pair()) return rc;
    FHD_CUDA_TRY(cudaEventRecord(e0, ctx->stream));
    for (int r = 0; r < TUNE_REPS; r++)
        if (int rc = pair()) return rc;
    FHD_CUDA_TRY(cudaEventRecord(e1, ctx->stream));
    FHD_CUDA_TRY(cudaEventSynchronize(e1));
    float ms = 0.f;
    FHD_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
    us = 1000.f * ms / TUNE_REPS;
    return 0;
}

template <typename T>
static int tune_levels_locked(fhd_ctx* ctx, Multigrid<T>& M, std::vector<T*>& scratch, cudaEvent_t ev[2]) {
    const int dim = ctx->dim;
    const int force = ctx->tune_mode >= 2 ? ctx->tune_mode - 2 : -1;
    // scratch unknowns, right-hand sides and second buffers: 3 dim arrays of
    // the largest level timed, zeroed
    auto get_scratch = [&](i64 nc) -> int {
        if (!scratch.empty()) return 0;
        for (int i = 0; i < 3 * dim; i++) {
            void* p = nullptr;
            FHD_CUDA_TRY(cudaMallocAsync(&p, (size_t)nc * sizeof(T), ctx->stream));
            scratch.push_back((T*)p);
            FHD_CUDA_TRY(cudaMemsetAsync(p, 0, (size_t)nc * sizeof(T), ctx->stream));
        }
        return 0;
    };
    const int lcs = stag_coarse_first(ctx, M), lcc = cc_coarse_first(ctx, M);
    const i64 nc_max = ctx->g0.nc;
    for (int l = 0; l < (int)M.s.size(); l++) {
        StagLevel<T>& L = M.s[l];
        L.plan = SmoothPlan();
        if (l >= lcs || !all_even(L.g) || ctx->p.stag_mg_smoother == 0) continue;
        const std::string key = tune_key(ctx, L.g, 0, (int)sizeof(T));
        auto it = g_tune.find(key);
        if (force < 0 && it != g_tune.end()) {
            L.plan = it->second;
            continue;
        }
        std::vector<SmoothPlan> cands = stag_cands(ctx, L);
        if (force >= 0) {
            L.plan = cands[(size_t)force < cands.size() ? force : 0];
            L.plan.ncand = (int)cands.size();
            continue;
        }
        auto im = g_tune_import.find(key);
        if (im != g_tune_import.end() && im->second < (int)cands.size()) {
            L.plan = cands[im->second];
            L.plan.ncand = (int)cands.size();
            L.plan.index = im->second;
            g_tune[key] = L.plan;
            continue;
        }
        if (int rc = get_scratch(nc_max)) return rc;
        StagLevel<T> S = L;  // scratch unknowns, the level's coefficients
        for (int c = 0; c < dim; c++) {
            S.phi[c] = scratch[c];
            S.tmp[c] = scratch[dim + c];
            S.rhs[c] = scratch[2 * dim + c];
        }
        if (!stag_aligned(S, dim)) continue;
        int best = -1;
        for (size_t i = 0; i < cands.size(); i++) {
            float us = 0.f;
            if (int rc = time_pairs(ctx, ev[0], ev[1], [&]() { return stag_smooths_planned(ctx, S, cands[i], 2); },
                                    us))
                return rc;
            cands[i].us = us;
            if (best < 0 || us < cands[best].us) best = (int)i;
        }
        L.plan = cands[best];
        L.plan.ncand = (int)cands.size();
        L.plan.index = best;
        g_tune[key] = L.plan;
    }
    for (int l = 0; l < (int)M.c.size(); l++) {
        CCLevel<T>& C = M.c[l];
        C.plan = SmoothPlan();
        if (l >= lcc || !all_even(C.g)) continue;
        const std::string key = tune_key(ctx, C.g, 1, (int)sizeof(T));
        auto it = g_tune.find(key);
        if (force < 0 && it != g_tune.end()) {
            C.plan = it->second;
            continue;
        }
        std::vector<SmoothPlan> cands = cc_cands(ctx, C);
        if (force >= 0) {
            C.plan = cands[(size_t)force < cands.size() ? force : 0];
            C.plan.ncand = (int)cands.size();
            continue;
        }
        auto im = g_tune_import.find(key);
        if (im != g_tune_import.end() && im->second < (int)cands.size()) {
            C.plan = cands[im->second];
            C.plan.ncand = (int)cands.size();
            C.plan.index = im->second;
            g_tune[key] = C.plan;
            continue;
        }
        if (int rc = get_scratch(nc_max)) return rc;
        CCLevel<T> S = C;
        S.phi = scratch[0];
        S.tmp = scratch[1];
        S.rhs = scratch[2];
        int best = -1;
        for (size_t i = 0; i < cands.size(); i++) {
            float us = 0.f;
            if (int rc = time_pairs(ctx, ev[0], ev[1], [&]() {
                    S.plan = cands[i];
                    return cc_smooths(ctx, S, 2);
                }, us))
                return rc;
            cands[i].us = us;
            if (best < 0 || us < cands[best].us) best = (int)i;
        }
        C.plan = cands[best];
        C.plan.ncand = (int)cands.size();
        C.plan.index = best;
        g_tune[key] = C.plan;
    }
    return 0;
}

template <typename T>
static int tune_levels(fhd_ctx* ctx) {
    Multigrid<T>& M = mg_of<T>(ctx);
    // (with walls the staggered levels smooth with the wall colours and the
    // pressure levels keep the fixed rules)
    if (ctx->tune_mode == 0 || ctx->has_walls) {
        for (auto& L : M.s) L.plan = SmoothPlan();
        for (auto& C : M.c) C.plan = SmoothPlan();
        return 0;
    }
    // inside a capture the plans of the last solve call stand
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(ctx->stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return 0;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    const bool prof = ctx->prof;
    const long long launches = ctx->launches;
    ctx->prof = false;
    std::vector<T*> scratch;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    int rc = 0;
    if (cudaEventCreate(&ev[0]) != cudaSuccess || cudaEventCreate(&ev[1]) != cudaSuccess) {
        set_last_error("autotuner: cudaEventCreate failed");
        rc = FHD_ERR_CUDA;
    }
    if (!rc) rc = tune_levels_locked(ctx, M, scratch, ev);
    for (T* p : scratch) cudaFreeAsync(p, ctx->stream);
    for (cudaEvent_t e : ev)
        if (e) cudaEventDestroy(e);
    ctx->prof = prof;
    ctx->launches = launches;
    return rc;
}

// levels lc..bottom of the pressure V-cycle in one CTA (phi of level lc:
// input when lc == 0, else zero; holds the result)
template <typename T>
static int cc_coarse(fhd_ctx* ctx, Multigrid<T>& M, int lc) {
    const int nl = (int)M.c.size();
    CCCoarseArgs<T> a;
    memset(&a, 0, sizeof a);
    a.nlev = nl - lc;
    a.load_phi = lc == 0;
    a.n_down = ctx->p.mg_nsmooths_down;
    a.n_up = ctx->p.mg_nsmooths_up;
    a.n_bottom = ctx->p.mg_nsmooths_bottom;
    a.phi = M.c[lc].phi;
    a.rhs = M.c[lc].rhs;
    size_t off = 0;
    for (int m = 0; m < a.nlev; m++) {
        const CCLevel<T>& C = M.c[lc + m];
        a.g[m] = C.g;
        a.A[m] = C.op();
        a.off[m] = (int)off;
        off += (size_t)3 * (size_t)C.g.nc;
    }
    const size_t smem = off * sizeof(T);
    int rc = 0;
    with_dim(ctx->dim, [&](auto D) {
        constexpr int DIM = decltype(D)::value;
        rc |= rb_allow_smem(k_cc_coarse<T, DIM>, smem);
        if (rc) return;
        k_cc_coarse<T, DIM><<<1, CS_THREADS, smem, ctx->stream>>>(a);
        rc |= post(ctx);
    });
    return rc;
}

// V-cycle from level l; levels from lc down run in the coarse kernel
template <typename T>
static int cc_vcycle(fhd_ctx* ctx, Multigrid<T>& M, int l, int lc) {
    const int nl = (int)M.c.size();
    CCLevel<T>& C = M.c[l];
    if (l == lc) return cc_coarse(ctx, M, lc);
    if (l == nl - 1) return cc_smooths(ctx, C, ctx->p.mg_nsmooths_bottom);
    {
        int rc = cc_smooths(ctx, C, ctx->p.mg_nsmooths_down);
        if (rc) return rc;
    }
    CCLevel<T>& D = M.c[l + 1];
    int rc = 0;
    with_dim(ctx->dim, [&](auto Dm) {
        constexpr int DIM = decltype(Dm)::value;
        k_cc_resid_restrict<T, DIM><<<cell_grid(D.g), cell_block(), 0, ctx->stream>>>(C.g, D.g, C.op(), C.phi, C.rhs,
                                                                                     D.rhs);
        rc |= post(ctx);
    });
    if (rc) return rc;
    if (l + 1 != lc) FHD_CUDA_TRY(cudaMemsetAsync(D.phi, 0, sizeof(T) * D.g.nc, ctx->stream));
    rc = cc_vcycle(ctx, M, l + 1, lc);
    if (rc) return rc;
    with_dim(ctx->dim, [&](auto Dm) {
        constexpr int DIM = decltype(Dm)::value;
        k_cc_prolong<T, DIM><<<cell_grid(D.g), cell_block(), 0, ctx->stream>>>(C.g, D.g, C.phi, D.phi);
        rc |= post(ctx);
    });
    if (rc) return rc;
    return cc_smooths(ctx, C, ctx->p.mg_nsmooths_up);
}

// Phi = 0, then mg_max_vcycles V-cycles on M.c[0].rhs
template <typename T>
static int cc_solve(fhd_ctx* ctx, Multigrid<T>& M) {
    CCLevel<T>& C = M.c[0];
    const i64 nc = C.g.nc;
    FHD_CUDA_TRY(cudaMemsetAsync(C.phi, 0, sizeof(T) * nc, ctx->stream));
    const int maxv = ctx->p.mg_max_vcycles;
    double r0 = 1.0;
    if (maxv > 1) {
        k_maxabs<T><<<flat_blocks(nc), RED_THREADS, 0, ctx->stream>>>(nc, C.rhs, slot(ctx, S_MG));
        FHD_POST(ctx);
        int rc = sync_scalars(ctx, S_MG, 1);
        if (rc) return rc;
        r0 = ctx->hscal[S_MG];
        if (r0 == 0.0) return 0;
    }
    const int lc = cc_coarse_first(ctx, M);
    for (int vc = 1; vc <= maxv; vc++) {
        int rc = cc_vcycle(ctx, M, 0, lc);
        if (rc) return rc;
        if (vc == maxv) break;
        with_dim(ctx->dim, [&](auto D) {
            constexpr int DIM = decltype(D)::value;
            k_cc_resid<T, DIM><<<cell_grid(C.g), cell_block(), 0, ctx->stream>>>(C.g, C.op(), C.phi, C.rhs, C.tmp);
            rc |= post(ctx);
        });
        if (rc) return rc;
        k_maxabs<T><<<flat_blocks(nc), RED_THREADS, 0, ctx->stream>>>(nc, C.tmp, slot(ctx, S_MG));
        FHD_POST(ctx);
        rc = sync_scalars(ctx, S_MG, 1);
        if (rc) return rc;
        if (ctx->hscal[S_MG] <= fmax(ctx->p.mg_rel_tol * r0, ctx->p.mg_abs_tol)) break;
    }
    ctx->vcycles += maxv;
    return 0;
}

// ---------------------------------------------------------------------
// apply_precon (apply_precon.f90:29-475); visc_schur_approx 0 (simple
// Schur complements) or 1 (visc_schur_complement, 538-685)
// ---------------------------------------------------------------------
template <typename T>
static int precon_T(fhd_ctx* ctx, CSVec<double> b, SVec<double> x) {
    Multigrid<T>& M = mg_of<T>(ctx);
    const int dim = ctx->dim;
    const i64 nc = ctx->g0.nc;
    const Grid g = ctx->g0;
    cudaStream_t st = ctx->stream;
    const int pt = ctx->p.precon_type, apt = pt < 0 ? -pt : pt;
    const int av = ctx->visc < 0 ? -ctx->visc : ctx->visc;
    const double theta = ctx->theta;
    const bool fp64 = std::is_same<T, double>::value;
    const int nb = flat_blocks(nc);
    const bool bfbt = ctx->p.visc_schur_approx != 0;
    if (apt < 1 || apt > 5 || (bfbt && av == 3)) {
        set_last_error(bfbt && av == 3 ? "apply_precon: visc_schur_approx needs |visc_type| 1 or 2 "
                                         "(inverse_diag_lap.f90 has no |visc_type| = 3)"
                                       : "apply_precon: unsupported precon_type");
        return FHD_ERR_UNSUPPORTED;
    }
    StagLevel<T>& L0 = M.s[0];
    // velocity unknowns of the multigrid: the FP64 output itself, or FP32
    // work arrays in the mixed preconditioner
    for (int c = 0; c < dim; c++) L0.phi[c] = fp64 ? (T*)x.c[c] : M.x_u[c];
    for (int c = 0; c < dim; c++) FHD_CUDA_TRY(cudaMemsetAsync(L0.phi[c], 0, sizeof(T) * nc, st));
    auto set_rhs_from_b = [&]() -> int {
        for (int c = 0; c < dim; c++) {
            if (fp64) {
                L0.rhs[c] = (T*)b.c[c];
            } else {
                k_copy_conv<T, double><<<nb, 256, 0, st>>>(nc, M.b_u[c], b.c[c], 1.0);
                FHD_POST(ctx);
                L0.rhs[c] = M.b_u[c];
            }
        }
        return 0;
    };
    auto phi_to_x = [&]() -> int {
        if (fp64) return 0;
        for (int c = 0; c < dim; c++) {
            k_copy_conv<double, T><<<nb, 256, 0, st>>>(nc, x.c[c], L0.phi[c], 1.0);
            FHD_POST(ctx);
        }
        return 0;
    };
    auto div_plus = [&](const double* bp) -> int {
        int rc = 0;
        with_dim(dim, [&](auto D) {
            constexpr int DIM = decltype(D)::value;
            k_div_plus<T, DIM><<<cell_grid(g), cell_block(), 0, st>>>(g, L0.phi[0], L0.phi[1], L0.phi[2], bp,
                                                                    M.c[0].rhs, (T)(1.0 / g.dx));
            rc |= post(ctx);
        });
        return rc;
    };
    auto schur = [&](int kind, int add_phi, int negate) -> int {
        int rc = 0;
        with_dim(dim, [&](auto D) {
            constexpr int DIM = decltype(D)::value;
            k_schur<T, DIM><<<cell_grid(g), cell_block(), 0, st>>>(g, M.c[0].op(), M.c[0].rhs, M.c[0].phi, ctx->beta,
                                                                 ctx->gamma, theta, av, kind, add_phi, negate,
                                                                 x.c[dim]);
            rc |= post(ctx);
        });
        return rc;
    };
    // visc_schur_complement (apply_precon.f90:538-685): x_p = Phi_mu2 (+
    // theta Phi), Phi_mu = L_mu^-1 mac_rhs, Phi_mu2 = L_mu^-1 D mu^-1 L
    // mu^-1 G Phi_mu; L_mu the pressure multigrid on the mu^-1 faces, L the
    // viscous operator without the alpha term
    auto visc_schur = [&](int add_phi, int negate) -> int {
        CCLevel<T>& C0 = M.c[0];
        int rc = 0;
        if (add_phi) FHD_CUDA_TRY(cudaMemcpyAsync(M.bf_phi, C0.phi, sizeof(T) * nc, cudaMemcpyDeviceToDevice, st));
        auto swap_coef = [&]() {
            for (auto& C : M.c)
                for (int c = 0; c < 3; c++) std::swap(C.a[c], C.amu[c]);
        };
        swap_coef();  // the pressure multigrid now runs on mu^-1
        rc = cc_solve(ctx, M);
        if (!rc) {
            StagOp<T> A = L0.op();
            A.alpha_scale = T(0);
            with_dim_visc(dim, ctx->visc, [&](auto D, auto V) {
                constexpr int DIM = decltype(D)::value, VISC = decltype(V)::value;
                k_grad_mul<T, DIM><<<cell_grid(g), cell_block(), 0, st>>>(
                    g, C0.phi, C0.a[0], C0.a[1], C0.a[2], M.bf_g[0], M.bf_g[1], M.bf_g[2], (T)(1.0 / g.dx));
                rc |= post(ctx);
                k_stag_apply<T, DIM, VISC><<<cell_grid(g), cell_block(), 0, st>>>(
                    g, A, M.bf_g[0], M.bf_g[1], M.bf_g[2], L0.tmp[0], L0.tmp[1], L0.tmp[2], nullptr, nullptr,
                    nullptr, 0);
                rc |= post(ctx);
                k_mul_faces<T><<<nb, 256, 0, st>>>(nc, DIM, L0.tmp[0], L0.tmp[1], L0.tmp[2], C0.a[0], C0.a[1],
                                                   C0.a[2]);
                rc |= post(ctx);
                k_div_plus<T, DIM><<<cell_grid(g), cell_block(), 0, st>>>(g, L0.tmp[0], L0.tmp[1], L0.tmp[2],
                                                                        nullptr, C0.rhs, (T)(1.0 / g.dx));
                rc |= post(ctx);
            });
        }
        if (!rc) rc = cc_solve(ctx, M);
        swap_coef();
        if (rc) return rc;
        k_bfbt_out<T><<<nb, 256, 0, st>>>(nc, x.c[dim], C0.phi, M.bf_phi, theta, add_phi, negate);
        FHD_POST(ctx);
        return 0;
    };
    // b_u - G x_p into the multigrid rhs (precon 3 and 5)
    auto rhs_minus_grad_xp = [&]() -> int {
        int rc = 0;
        with_dim(dim, [&](auto D) {
            constexpr int DIM = decltype(D)::value;
            k_sub_grad_T<T, DIM><<<cell_grid(g), cell_block(), 0, st>>>(g, b.c[0], b.c[1], DIM == 3 ? b.c[2] : nullptr,
                                                                      x.c[dim], M.b_u[0], M.b_u[1], M.b_u[2],
                                                                      1.0 / g.dx);
            rc |= post(ctx);
        });
        for (int c = 0; c < dim; c++) L0.rhs[c] = M.b_u[c];
        return rc;
    };
    int rc = 0;
    if (apt == 1) {
        if ((rc = set_rhs_from_b())) return rc;
        if ((rc = stag_mg_run(ctx, M))) return rc;
        if ((rc = div_plus(b.c[dim]))) return rc;
        if ((rc = cc_solve(ctx, M))) return rc;
        with_dim(dim, [&](auto D) {
            constexpr int DIM = decltype(D)::value;
            k_sub_wgrad<T, DIM><<<cell_grid(g), cell_block(), 0, st>>>(
                g, L0.phi[0], L0.phi[1], L0.phi[2], M.c[0].a[0], M.c[0].a[1], M.c[0].a[2], M.c[0].phi, x.c[0],
                x.c[1], DIM == 3 ? x.c[2] : nullptr, (T)(1.0 / g.dx));
            rc |= post(ctx);
        });
        // the pressure gradient is zero on wall faces: x_u keeps x_u* there (zero)
        if (!rc) rc = zero_walls<double>(ctx, g, x.c[0], x.c[1], dim == 3 ? x.c[2] : nullptr);
        if (rc) return rc;
        const int kind = (pt == 1 || theta == 0.0) ? 0 : 1;
        if ((rc = bfbt ? visc_schur(fabs(theta) > 0.0, 0) : schur(kind, 1, 0))) return rc;
    } else if (apt == 2 || apt == 5) {
        if ((rc = set_rhs_from_b())) return rc;
        if ((rc = stag_mg_run(ctx, M))) return rc;
        if ((rc = div_plus(b.c[dim]))) return rc;
        if (fabs(theta) > 0.0) {
            if ((rc = cc_solve(ctx, M))) return rc;
        }
        if ((rc = bfbt ? visc_schur(fabs(theta) > 0.0, (pt == -2 || pt == -5))
                       : schur(0, fabs(theta) > 0.0, (pt == -2 || pt == -5))))
            return rc;
        if (apt == 5) {
            if ((rc = rhs_minus_grad_xp())) return rc;
            if ((rc = stag_mg_run(ctx, M))) return rc;
        }
        if ((rc = phi_to_x())) return rc;
    } else if (apt == 3) {
        k_copy_conv<T, double><<<nb, 256, 0, st>>>(nc, M.c[0].rhs, b.c[dim], pt == -3 ? -1.0 : 1.0);
        FHD_POST(ctx);
        if (fabs(theta) > 0.0) {
            if ((rc = cc_solve(ctx, M))) return rc;
        }
        if ((rc = bfbt ? visc_schur(fabs(theta) > 0.0, 0) : schur(0, fabs(theta) > 0.0, 0))) return rc;
        if ((rc = rhs_minus_grad_xp())) return rc;
        if ((rc = stag_mg_run(ctx, M))) return rc;
        if ((rc = phi_to_x())) return rc;
    } else {  // 4
        if ((rc = set_rhs_from_b())) return rc;
        if ((rc = stag_mg_run(ctx, M))) return rc;
        const bool use_phi = fabs(theta) > 0.0;
        if (use_phi) {
            k_copy_conv<T, double><<<nb, 256, 0, st>>>(nc, M.c[0].rhs, b.c[dim], 1.0);
            FHD_POST(ctx);
            if ((rc = cc_solve(ctx, M))) return rc;
        } else if (bfbt) {
            // mac_rhs keeps its zero initial value when theta_alpha = 0
            FHD_CUDA_TRY(cudaMemsetAsync(M.c[0].rhs, 0, sizeof(T) * nc, st));
        }
        if (bfbt) {
            if ((rc = visc_schur(use_phi, 0))) return rc;
        } else {
            if (use_phi) {
                // blockdiag kernel reads Phi in FP64: stage it through x_p
                k_copy_conv<double, T><<<nb, 256, 0, st>>>(nc, x.c[dim], M.c[0].phi, 1.0);
                FHD_POST(ctx);
            }
            k_schur_blockdiag<<<nb, 256, 0, st>>>(nc, b.c[dim], ctx->beta, ctx->gamma, x.c[dim], theta,
                                                  use_phi ? 1 : 0, av, pt, x.c[dim]);
            FHD_POST(ctx);
        }
        if ((rc = phi_to_x())) return rc;
    }
    // null space: mean of p, and of u when theta_alpha = 0 and no wall is
    // no-slip, for the periodic directions -- apply_precon.f90:429-460
    k_sum<double><<<nb, RED_THREADS, 0, st>>>(nc, x.c[dim], slot(ctx, S_MEAN));
    FHD_POST(ctx);
    k_sub_mean<double><<<nb, 256, 0, st>>>(nc, x.c[dim], ctx->dscal + S_MEAN, (double)nc);
    FHD_POST(ctx);
    if (theta == 0.0 && !ctx->noslip) {
        for (int c = 0; c < dim; c++) {
            // the velocity means go for periodic directions only
            if (ctx->walls.lo[c] != 0) continue;
            k_sum<double><<<nb, RED_THREADS, 0, st>>>(nc, x.c[c], slot(ctx, S_MEAN + 1 + c));
            FHD_POST(ctx);
            k_sub_mean<double><<<nb, 256, 0, st>>>(nc, x.c[c], ctx->dscal + S_MEAN + 1 + c, (double)nc);
            FHD_POST(ctx);
        }
    }
    return 0;
}

int precon(fhd_ctx* ctx, CSVec<double> b, SVec<double> x) {
    if (ctx->prec == FHD_PREC_MIXED) return precon_T<float>(ctx, b, x);
    return precon_T<double>(ctx, b, x);
}

int stag_mg_solve_dev(fhd_ctx* ctx, double* const phi[], const double* const rhs[]) {
    const int dim = ctx->dim;
    const i64 nc = ctx->g0.nc;
    if (ctx->prec == FHD_PREC_MIXED) {
        Multigrid<float>& M = ctx->mg32;
        for (int c = 0; c < dim; c++) {
            k_copy_conv<float, double><<<flat_blocks(nc), 256, 0, ctx->stream>>>(nc, M.x_u[c], phi[c], 1.0);
            FHD_POST(ctx);
            k_copy_conv<float, double><<<flat_blocks(nc), 256, 0, ctx->stream>>>(nc, M.b_u[c], rhs[c], 1.0);
            FHD_POST(ctx);
            M.s[0].phi[c] = M.x_u[c];
            M.s[0].rhs[c] = M.b_u[c];
        }
        int rc = stag_mg_run(ctx, M);
        if (rc) return rc;
        for (int c = 0; c < dim; c++) {
            k_copy_conv<double, float><<<flat_blocks(nc), 256, 0, ctx->stream>>>(nc, phi[c], M.x_u[c], 1.0);
            FHD_POST(ctx);
        }
        return 0;
    }
    Multigrid<double>& M = ctx->mg64;
    for (int c = 0; c < dim; c++) {
        M.s[0].phi[c] = phi[c];
        M.s[0].rhs[c] = (double*)rhs[c];
    }
    return stag_mg_run(ctx, M);
}

// ---------------------------------------------------------------------
// apply_matrix (apply_matrix.f90:24-157), FP64 always
// ---------------------------------------------------------------------
int stokes_apply(fhd_ctx* ctx, CSVec<double> x, CSVec<double> rhs, SVec<double> out, int mode) {
    StagOp<double> A;
    for (int c = 0; c < 3; c++) {
        A.alpha[c] = ctx->alpha_fc[c];
        A.bed[c] = ctx->beta_ed[c];
    }
    A.alpha_scale = ctx->theta;
    A.beta = ctx->beta;
    A.gamma = ctx->gamma;
    A.q = 1.0 / (ctx->dx * ctx->dx);
    int rc = 0;
    if (ctx->has_walls) {
        with_dim_wall_visc(ctx->dim, ctx->visc, [&](auto D, auto V) {
            constexpr int DIM = decltype(D)::value, VISC = decltype(V)::value;
            k_stokes_apply_w<DIM, VISC><<<cell_grid(ctx->g0), cell_block(), 0, ctx->stream>>>(
                ctx->g0, ctx->walls, A, x, rhs, out, mode, 1.0 / ctx->dx);
            rc |= post(ctx);
        });
        return rc;
    }
    if (ctx->p.gmres_spatial_order == 4) {
        const double t1 = 1.0 / (12.0 * ctx->dx), t2 = 1.0 / (12.0 * ctx->dx * ctx->dx);
        if (ctx->dim == 2)
            k_stokes_apply4<2><<<cell_grid(ctx->g0), cell_block(), 0, ctx->stream>>>(ctx->g0, A, x, rhs, out, mode,
                                                                                   1.0 / ctx->dx, t1, t2);
        else
            k_stokes_apply4<3><<<cell_grid(ctx->g0), cell_block(), 0, ctx->stream>>>(ctx->g0, A, x, rhs, out, mode,
                                                                                   1.0 / ctx->dx, t1, t2);
        return post(ctx);
    }
    with_dim_visc(ctx->dim, ctx->visc, [&](auto D, auto V) {
        constexpr int DIM = decltype(D)::value, VISC = decltype(V)::value;
        k_stokes_apply<DIM, VISC><<<cell_grid(ctx->g0), cell_block(), 0, ctx->stream>>>(ctx->g0, A, x, rhs, out, mode,
                                                                                      1.0 / ctx->dx);
        rc |= post(ctx);
    });
    return rc;
}

// a bounded wait inside a kernel that ran out (the kernel set the context's
// error word and returned); cleared on read
int dev_err_check(fhd_ctx* ctx) {
    unsigned h = 0;
    FHD_CUDA_TRY(cudaMemcpyAsync(&h, ctx->dev_err, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
    FHD_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (h) {
        FHD_CUDA_TRY(cudaMemsetAsync(ctx->dev_err, 0, sizeof(unsigned), ctx->stream));
        set_last_error("a staging wait inside the fused smoother timed out");
        return FHD_ERR_CUDA;
    }
    return 0;
}

int sync_scalars(fhd_ctx* ctx, int first, int count) {
    FHD_CUDA_TRY(cudaMemcpyAsync(ctx->hscal + first, ctx->dscal + first, sizeof(double) * count,
                                 cudaMemcpyDeviceToHost, ctx->stream));
    FHD_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return 0;
}

// ---------------------------------------------------------------------
// preconditioner applications as CUDA graphs
// ---------------------------------------------------------------------
// Inside GMRES a preconditioner application is a fixed sequence of launches
// on the context stream with no host synchronisation (one V-cycle of each
// multigrid).  The first application for a given (b, x, prepared
// coefficients, theta) is captured into a graph; later ones replay it, one
// launch instead of a few hundred.  The values behind the pointers may
// change between replays (new coefficients, new right-hand sides); the key
// changes when a pointer or theta does.
static const size_t GRAPH_CACHE = 32;

static unsigned long long mix_key(unsigned long long h, unsigned long long v) {
    h ^= v + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2);
    return h;
}

static bool graphs_on(fhd_ctx* ctx) {
    if (ctx->p.stag_mg_max_vcycles > 1 || ctx->p.mg_max_vcycles > 1) return false;
    return ctx->graph_mode != 0;
}

static void drop_graph(fhd_ctx::PreconGraph& gr) {
    cudaGraphExecDestroy(gr.exec);
    if (gr.graph) cudaGraphDestroy(gr.graph);
}

void release_graphs(fhd_ctx* ctx) {
    for (auto& gr : ctx->graphs) drop_graph(gr);
    ctx->graphs.clear();
}

// launch a cached application: fresh events for its profiling nodes, the
// profiling totals and the launch counters it stands for
static int replay(fhd_ctx* ctx, fhd_ctx::PreconGraph& gr) {
    for (cudaGraphNode_t nd : gr.ev_nodes)
        FHD_CUDA_TRY(cudaGraphExecEventRecordNodeSetEvent(gr.exec, nd, prof_event(ctx)));
    FHD_CUDA_TRY(cudaGraphLaunch(gr.exec, ctx->stream));
    ctx->prof_bytes += gr.prof_bytes;
    ctx->prof_launches += gr.prof_launches;
    ctx->launches += gr.launches;
    ctx->vcycles += gr.vcycles;
    return 0;
}

// key of the prepared operator: coefficient pointers, theta and whether
// launches are being timed
static unsigned long long operator_key(fhd_ctx* ctx) {
    unsigned long long key = 1469598103934665603ull;
    for (int c = 0; c < 3; c++) {
        key = mix_key(key, (unsigned long long)(uintptr_t)ctx->alpha_fc[c]);
        key = mix_key(key, (unsigned long long)(uintptr_t)ctx->beta_ed[c]);
    }
    key = mix_key(key, (unsigned long long)(uintptr_t)ctx->beta);
    key = mix_key(key, (unsigned long long)(uintptr_t)ctx->gamma);
    unsigned long long tb;
    memcpy(&tb, &ctx->theta, sizeof(tb));
    key = mix_key(key, tb);
    key = mix_key(key, ctx->prof ? 1ull : 0ull);
    return key;
}

// Run fn() (a fixed sequence of launches and copies on ctx->stream with no
// host synchronisation) as a CUDA graph: the first call for a key captures
// it (thread-local: other threads' CUDA calls are unaffected), later calls
// replay it.  fn runs directly when graphs are off or the capture fails.
template <class F>
static int graphed(fhd_ctx* ctx, unsigned long long key, F&& fn) {
    if (!graphs_on(ctx)) return fn();
    ctx->graph_clock++;
    for (auto& gr : ctx->graphs) {
        if (gr.key != key) continue;
        gr.used = ctx->graph_clock;
        return replay(ctx, gr);
    }
    // the profiling events are made before the capture so that none is
    // created inside it
    if (ctx->prof)
        while (ctx->prof_ev.size() < ctx->prof_used + 512) {
            cudaEvent_t ev;
            FHD_CUDA_TRY(cudaEventCreate(&ev));
            ctx->prof_ev.push_back(ev);
        }
    const long long l0 = ctx->launches, pl0 = ctx->prof_launches;
    const int v0 = ctx->vcycles;
    const size_t pu0 = ctx->prof_used;
    const double pb0 = ctx->prof_bytes;
    if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return fn();
    }
    ctx->capturing = true;
    ctx->cap_fail = false;
    ctx->cap_nodes.clear();
    int rc = fn();
    ctx->capturing = false;
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
    cudaGraphExec_t exec = nullptr;
    if (!rc && e == cudaSuccess && graph && !ctx->cap_fail) e = cudaGraphInstantiate(&exec, graph, 0);
    fhd_ctx::PreconGraph gr;
    gr.key = key;
    gr.launches = ctx->launches - l0;
    gr.vcycles = ctx->vcycles - v0;
    gr.prof_launches = ctx->prof_launches - pl0;
    gr.prof_bytes = ctx->prof_bytes - pb0;
    gr.ev_nodes = ctx->cap_nodes;
    // nothing ran during the capture: undo its counts (the replay adds them)
    ctx->launches = l0;
    ctx->vcycles = v0;
    ctx->prof_launches = pl0;
    ctx->prof_bytes = pb0;
    ctx->prof_used = pu0;
    if (rc || e != cudaSuccess || !exec || ctx->cap_fail) {
        // not capturable here: run it directly
        cudaGetLastError();
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (rc) return rc;
        ctx->graph_mode = 0;
        return fn();
    }
    // the template graph stays alive while its event nodes are re-pointed
    if (gr.ev_nodes.empty()) {
        cudaGraphDestroy(graph);
        graph = nullptr;
    }
    gr.exec = exec;
    gr.graph = graph;
    gr.used = ctx->graph_clock;
    if (ctx->graphs.size() >= GRAPH_CACHE) {
        auto it = std::min_element(ctx->graphs.begin(), ctx->graphs.end(),
                                   [](const fhd_ctx::PreconGraph& a, const fhd_ctx::PreconGraph& b2) {
                                       return a.used < b2.used;
                                   });
        drop_graph(*it);
        ctx->graphs.erase(it);
    }
    ctx->graphs.push_back(gr);
    return replay(ctx, ctx->graphs.back());
}

static int precon_graphed(fhd_ctx* ctx, CSVec<double> b, SVec<double> x) {
    unsigned long long key = operator_key(ctx);
    for (int c = 0; c < 4; c++) {
        key = mix_key(key, (unsigned long long)(uintptr_t)b.c[c]);
        key = mix_key(key, (unsigned long long)(uintptr_t)x.c[c]);
    }
    return graphed(ctx, key, [&]() { return precon(ctx, b, x); });
}

// ---------------------------------------------------------------------
// gmres (gmres.f90:32-619)
// ---------------------------------------------------------------------
static SVec<double> svec(double* base, int dim, i64 nc) {
    SVec<double> v;
    for (int c = 0; c < 4; c++) v.c[c] = c <= dim ? base + (i64)c * nc : nullptr;
    return v;
}
static CSVec<double> csv(SVec<double> v) {
    CSVec<double> o;
    for (int c = 0; c < 4; c++) o.c[c] = v.c[c];
    return o;
}

static int wnorm2(fhd_ctx* ctx, CSVec<double> a, int slotid) {
    const i64 nc = ctx->g0.nc;
    const double wp = ctx->p.p_norm_weight;
    k_sdot<double, double><<<flat_blocks(nc), RED_THREADS, 0, ctx->stream>>>(nc, ctx->dim + 1, a, a, wp * wp,
                                                                          slot(ctx, slotid));
    return post(ctx);
}

int gmres_dev(fhd_ctx* ctx, CSVec<double> b, SVec<double> x, double* norm_pre_rhs, fhd_solve_stats* stout) {
    const int dim = ctx->dim, ncomp = dim + 1;
    const i64 nc = ctx->g0.nc;
    const fhd_gmres_params& p = ctx->p;
    const int m = p.gmres_max_inner;
    const double wp = p.p_norm_weight;
    cudaStream_t st = ctx->stream;
    const int nb = flat_blocks(nc);
    const i64 vstride = (i64)ncomp * nc;
    SVec<double> tmp = svec(ctx->tmp, dim, nc), r = svec(ctx->r, dim, nc), w = svec(ctx->w, dim, nc);
    auto V = [&](int k) { return svec(ctx->V + (i64)k * vstride, dim, nc); };  // 0-based
    fhd_solve_stats S;
    memset(&S, 0, sizeof(S));
    ctx->vcycles = 0;
    int rc;
    int status = 0;
    // |M^-1 b|
    if ((rc = precon_graphed(ctx, b, tmp))) return rc;
    if ((rc = wnorm2(ctx, csv(tmp), S_NRM))) return rc;
    if ((rc = wnorm2(ctx, b, S_NRM + 1))) return rc;
    if ((rc = sync_scalars(ctx, S_NRM, 2))) return rc;
    const double norm_pre_b = sqrt(ctx->hscal[S_NRM]);
    const double norm_b = sqrt(ctx->hscal[S_NRM + 1]);
    if (norm_pre_rhs) *norm_pre_rhs = norm_pre_b;
    S.norm_b = norm_b;
    S.norm_pre_b = norm_pre_b;
    if (norm_b <= p.gmres_abs_tol) {
        for (int c = 0; c <= dim; c++) FHD_CUDA_TRY(cudaMemsetAsync(x.c[c], 0, sizeof(double) * nc, st));
        if (stout) *stout = S;
        return 0;
    }
    std::vector<double> H((m + 2) * (m + 2), 0.0), cs(m + 2), sn(m + 2), s(m + 2), y(m + 2);
    auto Hh = [&](int i, int j) -> double& { return H[i * (m + 2) + j]; };
    int total_iter = 0, iter = 0, i_copy = 0;
    double norm_resid = 0, norm_init_resid = 0, norm_resid_Stokes = 0, norm_init_Stokes = 0, norm_resid_est = 0;
    for (;;) {
        // tmp = b - A x
        if ((rc = stokes_apply(ctx, csv(x), b, tmp, 1))) return rc;
        if ((rc = wnorm2(ctx, csv(tmp), S_NRM))) return rc;
        if ((rc = precon_graphed(ctx, csv(tmp), r))) return rc;
        if ((rc = wnorm2(ctx, csv(r), S_NRM + 1))) return rc;
        if ((rc = sync_scalars(ctx, S_NRM, 2))) return rc;
        norm_resid_Stokes = sqrt(ctx->hscal[S_NRM]);
        norm_resid = sqrt(ctx->hscal[S_NRM + 1]);
        if (iter == 0) {
            norm_init_Stokes = norm_resid_Stokes;
            norm_init_resid = norm_resid;
            norm_resid_est = norm_resid;
        }
        if (total_iter >= p.gmres_max_iter) {
            status = FHD_WARN_NOT_CONVERGED_MAXITER;
            break;
        } else if (total_iter >= p.gmres_min_iter) {
            if (norm_resid <= p.gmres_rel_tol * fmin(norm_pre_b, norm_init_resid)) {
                if (norm_resid_Stokes >= 10 * p.gmres_rel_tol * fmin(norm_b, norm_init_Stokes))
                    status = FHD_WARN_TRUE_RESID;
                break;
            } else if (norm_resid <= p.gmres_abs_tol) {
                break;
            }
        }
        if (iter >= p.gmres_max_outer) {
            status = FHD_WARN_NOT_CONVERGED_OUTER;
            break;
        }
        iter++;
        k_scale_div<<<nb, 256, 0, st>>>(nc, ncomp, V(0), csv(r), norm_resid);
        FHD_POST(ctx);
        std::fill(s.begin(), s.end(), 0.0);
        s[1] = norm_resid;
        for (int i = 1; i <= m; i++) {
            total_iter++;
            i_copy = i;
            // the iteration's launches -- A v_{i-1}, the preconditioner,
            // modified Gram-Schmidt with device-resident coefficients, the
            // normalisation -- and the copy of the new Hessenberg column to
            // the host: in graph mode 2 replayed as one graph per i, else
            // launched one by one around the preconditioner's graph
            const bool igraph = ctx->graph_mode == 2;
            auto body = [&]() -> int {
                int r2;
                if ((r2 = stokes_apply(ctx, csv(V(i - 1)), csv(V(i - 1)), tmp, 0))) return r2;
                if ((r2 = igraph ? precon(ctx, csv(tmp), w) : precon_graphed(ctx, csv(tmp), w))) return r2;
                for (int k = 1; k <= i; k++) {
                    CSVec<double> none;
                    for (int c = 0; c < 4; c++) none.c[c] = nullptr;
                    k_mgs<<<nb, RED_THREADS, 0, st>>>(nc, ncomp, w, k > 1 ? csv(V(k - 2)) : none,
                                                      k > 1 ? ctx->dscal + S_H + k - 1 : nullptr, csv(V(k - 1)),
                                                      wp * wp, slot(ctx, S_H + k));
                    FHD_POST(ctx);
                }
                {
                    CSVec<double> none;
                    for (int c = 0; c < 4; c++) none.c[c] = nullptr;
                    k_mgs<<<nb, RED_THREADS, 0, st>>>(nc, ncomp, w, csv(V(i - 1)), ctx->dscal + S_H + i, none,
                                                      wp * wp, slot(ctx, S_NRM));
                    FHD_POST(ctx);
                }
                k_scale_by_norm<<<nb, 256, 0, st>>>(nc, ncomp, V(i), csv(w), ctx->dscal + S_NRM);
                FHD_POST(ctx);
                FHD_CUDA_TRY(cudaMemcpyAsync(ctx->hscal + S_H + 1, ctx->dscal + S_H + 1, sizeof(double) * i,
                                             cudaMemcpyDeviceToHost, st));
                FHD_CUDA_TRY(cudaMemcpyAsync(ctx->hscal + S_NRM, ctx->dscal + S_NRM, sizeof(double),
                                             cudaMemcpyDeviceToHost, st));
                return 0;
            };
            const unsigned long long ikey =
                mix_key(mix_key(operator_key(ctx), 0x61726e6f6c6469ull), (unsigned long long)i);
            if ((rc = igraph ? graphed(ctx, ikey, body) : body())) return rc;
            FHD_CUDA_TRY(cudaStreamSynchronize(st));
            for (int k = 1; k <= i; k++) Hh(k, i) = ctx->hscal[S_H + k];
            Hh(i + 1, i) = sqrt(ctx->hscal[S_NRM]);
            if (Hh(i + 1, i) == 0.0) {
                set_last_error("gmres: error in orthogonalization");
                return FHD_ERR_ORTHO_BREAKDOWN;
            }
            // least_squares + rotmat (gmres.f90:531-597)
            for (int k = 1; k <= i - 1; k++) {
                double t = cs[k] * Hh(k, i) + sn[k] * Hh(k + 1, i);
                Hh(k + 1, i) = -sn[k] * Hh(k, i) + cs[k] * Hh(k + 1, i);
                Hh(k, i) = t;
            }
            {
                double a = Hh(i, i), bb = Hh(i + 1, i);
                if (bb == 0.0) {
                    cs[i] = 1.0;
                    sn[i] = 0.0;
                } else if (fabs(bb) > fabs(a)) {
                    double t = a / bb;
                    sn[i] = 1.0 / sqrt(1.0 + t * t);
                    cs[i] = t * sn[i];
                } else {
                    double t = bb / a;
                    cs[i] = 1.0 / sqrt(1.0 + t * t);
                    sn[i] = t * cs[i];
                }
                double t = cs[i] * s[i];
                s[i + 1] = -sn[i] * s[i];
                s[i] = t;
                Hh(i, i) = cs[i] * Hh(i, i) + sn[i] * Hh(i + 1, i);
                Hh(i + 1, i) = 0.0;
            }
            norm_resid_est = fabs(s[i + 1]);
            if (total_iter >= p.gmres_max_iter) break;
            else if (total_iter >= p.gmres_min_iter) {
                if (norm_resid_est <= p.gmres_rel_tol * fmin(norm_pre_b, norm_init_resid) ||
                    norm_resid_est <= p.gmres_abs_tol)
                    break;
            }
        }
        // SolveUTriangular (gmres.f90:599-619) and update_sol
        {
            const int k = i_copy - 1;
            y[k + 1] = s[k + 1] / Hh(k + 1, k + 1);
            for (int ii = k; ii >= 1; ii--) {
                double acc = 0.0;
                for (int jj = ii + 1; jj <= k + 1; jj++) acc += Hh(ii, jj) * y[jj];
                y[ii] = (s[ii] - acc) / Hh(ii, ii);
            }
            for (int it = 1; it <= i_copy; it++) ctx->hscal[S_Y + it - 1] = y[it];
            FHD_CUDA_TRY(cudaMemcpyAsync(ctx->dscal + S_Y, ctx->hscal + S_Y, sizeof(double) * i_copy,
                                         cudaMemcpyHostToDevice, st));
            k_update_sol<<<nb, 256, 0, st>>>(nc, ncomp, x, ctx->V, vstride, ctx->dscal + S_Y, i_copy);
            FHD_POST(ctx);
            // the staged y must not be overwritten before the copy ran
            FHD_CUDA_TRY(cudaStreamSynchronize(st));
        }
    }
    if ((rc = dev_err_check(ctx))) return rc;
    S.outer_iters = iter;
    S.total_iters = total_iter;
    S.vcycles = ctx->vcycles;
    S.status = status;
    S.norm_init_resid = norm_init_resid;
    S.norm_resid = norm_resid;
    S.norm_resid_Stokes = norm_resid_Stokes;
    S.norm_init_Stokes = norm_init_Stokes;
    S.norm_resid_est = norm_resid_est;
    if (stout) *stout = S;
    return status;
}

}  // namespace fhd

using namespace fhd;

// =====================================================================
// C ABI: context and device-pointer entry points
// =====================================================================
extern "C" {

void fhd_gmres_params_default(fhd_gmres_params* p) {
    // probin_gmres_init defaults (probin_gmres.f90:122-163)
    memset(p, 0, sizeof(*p));
    p->precon_type = 1;
    p->visc_schur_approx = 0;
    p->p_norm_weight = 1.0;
    p->scale_factor = 1.0;
    p->mg_verbose = 0;
    p->cg_verbose = 0;
    p->mg_max_vcycles = 1;
    p->mg_minwidth = 2;
    p->mg_bottom_solver = 4;
    p->mg_nsmooths_down = 2;
    p->mg_nsmooths_up = 2;
    p->mg_nsmooths_bottom = 8;
    p->mg_max_bottom_nlevels = 10;
    p->mg_rel_tol = 1e-9;
    p->mg_abs_tol = 1e-14;
    p->stag_mg_verbosity = 0;
    p->stag_mg_max_vcycles = 1;
    p->stag_mg_minwidth = 2;
    p->stag_mg_bottom_solver = 4;
    p->stag_mg_nsmooths_down = 2;
    p->stag_mg_nsmooths_up = 2;
    p->stag_mg_nsmooths_bottom = 8;
    p->stag_mg_max_bottom_nlevels = 10;
    p->stag_mg_omega = 1.0;
    p->stag_mg_smoother = 1;
    p->stag_mg_rel_tol = 1e-9;
    p->gmres_rel_tol = 1e-9;
    p->gmres_abs_tol = 0.0;
    p->gmres_verbose = 1;
    p->gmres_max_outer = 20;
    p->gmres_max_inner = 5;
    p->gmres_max_iter = 100;
    p->gmres_min_iter = 1;
    p->gmres_spatial_order = 2;
}

const char* fhd_status_string(int s) {
    switch (s) {
        case FHD_OK: return "ok";
        case FHD_WARN_NOT_CONVERGED_MAXITER: return "GMRES did not converge in max number of total inner iterations";
        case FHD_WARN_NOT_CONVERGED_OUTER: return "GMRES did not converge in max number of outer iterations";
        case FHD_WARN_TRUE_RESID: return "gmres may not have converged (true residual above tolerance)";
        case FHD_ERR_BAD_ARG: return "bad argument";
        case FHD_ERR_BAD_GHOSTS: return "x_u and x_p need at least 1 ghost cell";
        case FHD_ERR_DX_NOT_ISOTROPIC: return "only dx=dy(=dz) is supported";
        case FHD_ERR_ORTHO_BREAKDOWN: return "gmres: error in orthogonalization";
        case FHD_ERR_UNSUPPORTED: return "unsupported option";
        case FHD_ERR_NONFINITE: return "non-finite value";
        case FHD_ERR_OOM: return "out of device memory";
        case FHD_ERR_CUDA: return g_last_error.empty() ? "CUDA error" : g_last_error.c_str();
        case FHD_ERR_NO_DEVICE: return "no CUDA device";
    }
    return "unknown status";
}

const char* fhd_last_error(void) { return g_last_error.c_str(); }

static int ctx_create(int dim, const int n_cells[3], const int max_grid_size[3], const double dx[3], int visc_type,
                      const fhd_gmres_params* params, int precision_mode, fhd_ctx** out);

int fhd_ctx_create(int dim, const int n_cells[3], const double dx[3], int visc_type, const fhd_gmres_params* params,
                   int precision_mode, fhd_ctx** out) {
    return ctx_create(dim, n_cells, nullptr, dx, visc_type, params, precision_mode, out);
}

int fhd_ctx_create_bc(int dim, const int n_cells[3], const int max_grid_size[3], const int bc_lo[3],
                      const int bc_hi[3], const double dx[3], int visc_type, const fhd_gmres_params* params,
                      int precision_mode, fhd_ctx** out) {
    if (!out || !n_cells || !max_grid_size || !bc_lo || !bc_hi || (dim != 2 && dim != 3)) return FHD_ERR_BAD_ARG;
    *out = nullptr;
    Walls W = {{0, 0, 0}, {0, 0, 0}};
    bool any = false, noslip = false, res = false;
    // reservoirs are walls for everything the context's solves see
    // (refuse_reservoirs)
    auto sign = [&res](int code, int& w) {
        if (code == FHD_BC_PERIODIC) w = 0;
        else if (code == FHD_BC_NO_SLIP_WALL || code == FHD_BC_NO_SLIP_RESERVOIR) w = -1;
        else if (code == FHD_BC_SLIP_WALL || code == FHD_BC_SLIP_RESERVOIR) w = 1;
        else return false;
        res = res || code == FHD_BC_NO_SLIP_RESERVOIR || code == FHD_BC_SLIP_RESERVOIR;
        return true;
    };
    for (int d = 0; d < dim; d++) {
        if (!sign(bc_lo[d], W.lo[d]) || !sign(bc_hi[d], W.hi[d])) {
            set_last_error("fhd_ctx_create_bc: bc codes -1 (periodic), 100 (no-slip wall), 200 (slip wall), 101 "
                           "and 201 (reservoirs) are built; other codes are not");
            return FHD_ERR_UNSUPPORTED;
        }
        if ((W.lo[d] == 0) != (W.hi[d] == 0)) {
            set_last_error("fhd_ctx_create_bc: a direction is periodic on both sides or on neither");
            return FHD_ERR_BAD_ARG;
        }
        any = any || W.lo[d] != 0;
        noslip = noslip || W.lo[d] < 0 || W.hi[d] < 0;
        if (max_grid_size[d] < 1) return FHD_ERR_BAD_ARG;
        if (max_grid_size[d] < n_cells[d] && n_cells[d] % max_grid_size[d] != 0) {
            set_last_error("fhd_ctx_create_bc: max_grid_size must divide n_cells (boxes of equal size)");
            return FHD_ERR_UNSUPPORTED;
        }
    }
    if (any) {
        fhd_gmres_params p;
        if (params) p = *params;
        else fhd_gmres_params_default(&p);
        bool boxes = false;
        for (int d = 0; d < dim; d++) boxes = boxes || max_grid_size[d] < n_cells[d];
        if (visc_type < 1 || p.precon_type != 1 || p.visc_schur_approx != 0 || p.stag_mg_smoother == 0 ||
            p.gmres_spatial_order != 2 || boxes) {
            set_last_error("fhd_ctx_create_bc: walls are built for visc_type 1, 2 or 3, precon_type 1 without the BFBt "
                           "Schur complement, the colour smoother, second order and one box");
            return FHD_ERR_UNSUPPORTED;
        }
    }
    const int rc = ctx_create(dim, n_cells, max_grid_size, dx, visc_type, params, precision_mode, out);
    if (rc == FHD_OK && any) {
        fhd_ctx* c = *out;
        c->walls = W;
        c->has_walls = true;
        c->noslip = noslip;
        c->reservoirs = res;
        const int r2 = c->prec == FHD_PREC_MIXED ? wall_diag<float>(c) : wall_diag<double>(c);
        if (r2 != FHD_OK) {
            fhd_ctx_destroy(c);
            *out = nullptr;
            return r2;
        }
    }
    return rc;
}

static int ctx_create(int dim, const int n_cells[3], const int max_grid_size[3], const double dx[3], int visc_type,
                      const fhd_gmres_params* params, int precision_mode, fhd_ctx** out) {
    if (!out || !n_cells || !dx || (dim != 2 && dim != 3)) return FHD_ERR_BAD_ARG;
    *out = nullptr;
    if (visc_type == 0 || visc_type < -3 || visc_type > 3) return FHD_ERR_BAD_ARG;
    for (int d = 0; d < dim; d++)
        if (n_cells[d] < 2) return FHD_ERR_BAD_ARG;
    for (int d = 1; d < dim; d++)
        if (dx[d] >= (1.0 + 1e-12) * dx[0] || dx[d] <= (1.0 - 1e-12) * dx[0]) return FHD_ERR_DX_NOT_ISOTROPIC;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return FHD_ERR_NO_DEVICE;
    fhd_ctx* c = new fhd_ctx();
    c->dim = dim;
    for (int d = 0; d < 3; d++) c->n[d] = (d < dim) ? n_cells[d] : 1;
    for (int d = 0; d < 3; d++) c->mgs[d] = (max_grid_size && d < dim) ? max_grid_size[d] : 0;
    c->dx = dx[0];
    c->visc = visc_type;
    c->prec = precision_mode == FHD_PREC_MIXED ? FHD_PREC_MIXED : FHD_PREC_FP64;
    if (params) c->p = *params;
    else fhd_gmres_params_default(&c->p);
    if (c->p.gmres_max_inner < 1 || c->p.gmres_max_inner > 60) {
        delete c;
        return FHD_ERR_UNSUPPORTED;
    }
    // gmres_spatial_order 4: stag_applyop_4o exists for visc_type 1 only
    // (stag_applyop.f90:1355, 1506)
    if (c->p.gmres_spatial_order != 2 && !(c->p.gmres_spatial_order == 4 && visc_type == 1)) {
        set_last_error("gmres_spatial_order 4 supports visc_type 1 only; other orders are not defined");
        delete c;
        return FHD_ERR_UNSUPPORTED;
    }
    c->m = c->p.gmres_max_inner;
    c->g0 = make_grid(dim, c->n, c->dx);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return FHD_ERR_CUDA;
    }
    c->own = c->stream;
    c->arena.stream = &c->stream;
    int rc = (c->prec == FHD_PREC_MIXED) ? build_mg(c, c->mg32) : build_mg(c, c->mg64);
    const i64 nc = c->g0.nc;
    const i64 sv = (i64)(dim + 1) * nc;
    if (!rc) {
        c->V = c->arena.alloc<double>(sv * (c->m + 1));
        c->r = c->arena.alloc<double>(sv);
        c->w = c->arena.alloc<double>(sv);
        c->tmp = c->arena.alloc<double>(sv);
        c->xs = c->arena.alloc<double>(sv);
        c->red_partials = c->arena.alloc<double>(RED_MAX_BLOCKS);
        c->red_counter = (unsigned*)c->arena.alloc<double>(1);
        c->dscal = c->arena.alloc<double>(NSCAL);
        c->dev_err = (unsigned*)c->arena.alloc<double>(1);
        if (!c->V || !c->r || !c->w || !c->tmp || !c->xs || !c->red_partials || !c->red_counter || !c->dscal ||
            !c->dev_err)
            rc = FHD_ERR_OOM;
    }
    if (!rc && !(c->hscal = pinned_scalars_acquire())) rc = FHD_ERR_OOM;
    if (!rc && cudaMemsetAsync(c->red_counter, 0, sizeof(double), c->stream) != cudaSuccess) rc = FHD_ERR_CUDA;
    if (!rc && cudaMemsetAsync(c->dev_err, 0, sizeof(double), c->stream) != cudaSuccess) rc = FHD_ERR_CUDA;
    if (!rc) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&c->smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&c->smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess)
            rc = FHD_ERR_CUDA;
    }
    if (!rc && cudaStreamSynchronize(c->stream) != cudaSuccess) rc = FHD_ERR_CUDA;
    if (rc) {
        fhd_ctx_destroy(c);
        return rc;
    }
    *out = c;
    return FHD_OK;
}

void fhd_host_path_release(fhd_ctx* ctx);
void fhd_mass_release(fhd_ctx* ctx);

int fhd_ctx_destroy(fhd_ctx* c) {
    if (!c) return FHD_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    // free on the context's own stream: a caller's stream may not outlive it
    if (c->own) c->stream = c->own;
    release_graphs(c);
    fhd_host_path_release(c);
    fhd_mass_release(c);
    c->arena.release();
    for (cudaEvent_t e : c->prof_ev) cudaEventDestroy(e);
    c->prof_ev.clear();
    pinned_scalars_release(c->hscal);
    if (c->own) cudaStreamDestroy(c->own);
    delete c;
    return FHD_OK;
}

void* fhd_ctx_stream(fhd_ctx* c) { return c ? (void*)c->stream : nullptr; }

int fhd_ctx_set_stream(fhd_ctx* c, void* s) {
    if (!c) return FHD_ERR_BAD_ARG;
    c->stream = s ? (cudaStream_t)s : c->own;
    return FHD_OK;
}

long long fhd_ctx_kernel_launches(fhd_ctx* c) { return c ? c->launches : 0; }

int fhd_ctx_profile(fhd_ctx* c, int enable) {
    if (!c) return FHD_ERR_BAD_ARG;
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return FHD_ERR_CUDA;
    c->prof = enable != 0;
    c->prof_used = 0;
    c->prof_bytes = 0.0;
    c->prof_launches = 0;
    return FHD_OK;
}

int fhd_ctx_profile_read(fhd_ctx* c, long long* launches, double* ms, double* bytes) {
    if (!c) return FHD_ERR_BAD_ARG;
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return FHD_ERR_CUDA;
    double t = 0.0;
    for (size_t i = 0; i + 1 < c->prof_used; i += 2) {
        float m = 0.f;
        if (cudaEventElapsedTime(&m, c->prof_ev[i], c->prof_ev[i + 1]) != cudaSuccess) return FHD_ERR_CUDA;
        t += m;
    }
    if (launches) *launches = c->prof_launches;
    if (ms) *ms = t;
    if (bytes) *bytes = c->prof_bytes;
    return FHD_OK;
}

int fhd_ctx_set_coarse(fhd_ctx* c, int mode) {
    if (!c || mode < -1 || mode > 1) return FHD_ERR_BAD_ARG;
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return FHD_ERR_CUDA;
    // captured preconditioner graphs hold the other launch sequence
    release_graphs(c);
    c->coarse_mode = mode;
    return FHD_OK;
}

int fhd_ctx_set_fused(fhd_ctx* c, int mode) {
    if (!c || mode < -1 || mode > 1) return FHD_ERR_BAD_ARG;
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return FHD_ERR_CUDA;
    // captured preconditioner graphs hold the other launch sequence
    release_graphs(c);
    c->fused_mode = mode;
    return FHD_OK;
}

int fhd_ctx_set_wall_speed(fhd_ctx* c, const double wallspeed_lo[6], const double wallspeed_hi[6]) {
    if (!c || !wallspeed_lo || !wallspeed_hi) return FHD_ERR_BAD_ARG;
    double v[2][6];
    bool any = false;
    for (int side = 0; side < 2; side++)
        for (int d = 0; d < 3; d++)
            for (int t = 0; t < 2; t++) {
                const int q = t + 2 * d;
                const double s = side ? wallspeed_hi[q] : wallspeed_lo[q];
                const int w = side ? c->walls.hi[d] : c->walls.lo[d];
                // only the speeds of this context's walls count (a periodic
                // side keeps its speed unused, as in the reference)
                const bool used = d < c->dim && t < c->dim - 1 && w != 0;
                if (used && s != 0.0 && w > 0) {
                    set_last_error("fhd_ctx_set_wall_speed: a slip wall takes no speed (its value is a traction)");
                    return FHD_ERR_UNSUPPORTED;
                }
                if (used && !std::isfinite(s)) return FHD_ERR_BAD_ARG;
                v[side][q] = used ? s : 0.0;
                any = any || v[side][q] != 0.0;
            }
    memcpy(c->wall_speed, v, sizeof(v));
    c->moving_walls = any;
    return FHD_OK;
}

int fhd_ctx_set_tune(fhd_ctx* c, int mode) {
    if (!c || mode < -1 || mode > 64) return FHD_ERR_BAD_ARG;
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return FHD_ERR_CUDA;
    release_graphs(c);
    c->tune_mode = mode;
    return FHD_OK;
}

long long fhd_tune_export(char* buf, long long len) {
    std::string out;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        std::map<std::string, int> all = g_tune_import;
        for (const auto& kv : g_tune)
            if (kv.second.index >= 0) all[kv.first] = kv.second.index;
        for (const auto& kv : all) out += kv.first + " " + std::to_string(kv.second) + "\n";
    }
    const long long need = (long long)out.size() + 1;
    if (buf && len > 0) {
        const long long n = need <= len ? need - 1 : len - 1;
        memcpy(buf, out.data(), (size_t)n);
        buf[n] = '\0';
    }
    return need;
}

int fhd_tune_import(const char* text) {
    if (!text) return FHD_ERR_BAD_ARG;
    std::map<std::string, int> got;
    const char* p = text;
    while (*p) {
        const char* e = strchr(p, '\n');
        const std::string line(p, e ? (size_t)(e - p) : strlen(p));
        p = e ? e + 1 : p + line.size();
        if (line.empty()) continue;
        const size_t sp = line.find(' ');
        if (sp == std::string::npos || sp == 0 || line.find(' ', sp + 1) != std::string::npos)
            return FHD_ERR_BAD_ARG;
        const std::string key = line.substr(0, sp), num = line.substr(sp + 1);
        if (num.empty() || num.size() > 4 || num.find_first_not_of("0123456789") != std::string::npos)
            return FHD_ERR_BAD_ARG;
        // version:device:which:element size:dim:visc_type:extents:SMs:shared
        // memory per block (opt-in):per SM, as the tuner writes them
        int ver, dev, elem, dim, visc, n0, n1, n2, sms, optin, smsm;
        char which;
        if (sscanf(key.c_str(), "v%d:%d:%c:%d:%d:%d:%dx%dx%d:%d:%d:%d", &ver, &dev, &which, &elem, &dim, &visc, &n0,
                   &n1, &n2, &sms, &optin, &smsm) != 12 ||
            (which != 's' && which != 'c') || (elem != 4 && elem != 8) || (dim != 2 && dim != 3))
            return FHD_ERR_BAD_ARG;
        // a line of another candidate-list version is well formed but names
        // plans of other lists: it is skipped
        if (ver != TUNE_CANDS_VERSION) continue;
        got[key] = atoi(num.c_str());
    }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (const auto& kv : got) g_tune_import[kv.first] = kv.second;
    return (int)got.size();
}

long long fhd_tune_key(int which, int dim, const int n_cells[3], int precision_mode, int visc_type, int sms,
                       int smem_optin, int smem_sm, int device, char* buf, long long len) {
    if ((which != 0 && which != 1) || (dim != 2 && dim != 3) || !n_cells || sms < 1 || smem_optin < 1 ||
        smem_sm < 1 || device < 0)
        return FHD_ERR_BAD_ARG;
    int n[3] = {n_cells[0], n_cells[1], dim == 3 ? n_cells[2] : 1};
    const std::string k = tune_key_of(device, which, precision_mode == FHD_PREC_MIXED ? 4 : 8, dim, visc_type, n, sms,
                                      smem_optin, smem_sm);
    const long long need = (long long)k.size() + 1;
    if (buf && len > 0) {
        const long long m = need <= len ? need - 1 : len - 1;
        memcpy(buf, k.data(), (size_t)m);
        buf[m] = '\0';
    }
    return need;
}

int fhd_tune_candidates(int which, int dim, const int n_cells[3], int precision_mode, int visc_type, int sms,
                        int smem_optin, int smem_sm, int* out, int max_out) {
    if ((which != 0 && which != 1) || (dim != 2 && dim != 3) || !n_cells || sms < 1 || smem_optin < 1 ||
        max_out < 0 || (max_out > 0 && !out))
        return FHD_ERR_BAD_ARG;
    for (int d = 0; d < dim; d++)
        if (n_cells[d] < 2) return FHD_ERR_BAD_ARG;
    fhd_ctx c;  // only the fields the candidate lists read
    c.dim = dim;
    c.visc = visc_type;
    c.sms = sms;
    c.smem_optin = smem_optin;
    c.smem_sm = smem_sm;
    const Grid g = make_grid(dim, n_cells, 1.0);
    std::vector<SmoothPlan> v;
    const bool f32 = precision_mode == FHD_PREC_MIXED;
    if (which == 0) {
        if (f32) {
            StagLevel<float> L;
            L.g = g;
            v = stag_cands(&c, L);
        } else {
            StagLevel<double> L;
            L.g = g;
            v = stag_cands(&c, L);
        }
    } else {
        if (f32) {
            CCLevel<float> C;
            C.g = g;
            v = cc_cands(&c, C);
        } else {
            CCLevel<double> C;
            C.g = g;
            v = cc_cands(&c, C);
        }
    }
    for (int i = 0; i < (int)v.size() && i < max_out; i++) {
        const SmoothPlan& P = v[i];
        int* o = out + 7 * i;
        o[0] = P.kind;
        o[1] = P.kind == 0 ? P.bx : P.kind == 1 ? P.rb.TX : g.n[0];
        o[2] = P.kind == 0 ? P.by : P.kind == 1 ? P.rb.TY : P.rbx.TY;
        o[3] = P.kind == 1 ? P.rb.chunks : P.kind == 2 ? P.rbx.chunks : 0;
        o[4] = P.kind == 2 ? P.rbx.per_sm : 1;
        o[5] = P.kind == 2 ? (int)P.rbx.smem : 0;
        o[6] = P.kind == 0 ? P.bx * P.by : P.kind == 1 ? P.rb.threads : P.rbx.threads;
    }
    return (int)v.size();
}

int fhd_ctx_tune_info(fhd_ctx* c, int which, int level, int* kind, int* ncand, double* pair_us, int shape[5]) {
    if (!c || (which != 0 && which != 1) || level < 0) return FHD_ERR_BAD_ARG;
    const SmoothPlan* P = nullptr;
    if (c->prec == FHD_PREC_MIXED) {
        if (which == 0 && level < (int)c->mg32.s.size()) P = &c->mg32.s[level].plan;
        if (which == 1 && level < (int)c->mg32.c.size()) P = &c->mg32.c[level].plan;
    } else {
        if (which == 0 && level < (int)c->mg64.s.size()) P = &c->mg64.s[level].plan;
        if (which == 1 && level < (int)c->mg64.c.size()) P = &c->mg64.c[level].plan;
    }
    if (!P) return FHD_ERR_BAD_ARG;
    if (kind) *kind = P->kind;
    if (ncand) *ncand = P->ncand;
    if (pair_us) *pair_us = P->us;
    if (shape) {
        shape[0] = P->kind == 0 ? P->bx : P->kind == 1 ? P->rb.TX : P->kind == 2 ? c->n[0] : 0;
        shape[1] = P->kind == 0 ? P->by : P->kind == 1 ? P->rb.TY : P->kind == 2 ? P->rbx.TY : 0;
        shape[2] = P->kind == 1 ? P->rb.chunks : P->kind == 2 ? P->rbx.chunks : 0;
        shape[3] = P->kind == 2 ? P->rbx.per_sm : P->kind >= 0 ? 1 : 0;
        shape[4] = P->kind == 0 ? P->bx * P->by : P->kind == 1 ? P->rb.threads : P->kind == 2 ? P->rbx.threads : 0;
    }
    return FHD_OK;
}

int fhd_ctx_set_graphs(fhd_ctx* c, int mode) {
    if (!c || mode < -1 || mode > 2) return FHD_ERR_BAD_ARG;
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return FHD_ERR_CUDA;
    c->graph_mode = mode;
    if (mode == 0) release_graphs(c);
    return FHD_OK;
}

unsigned long long fhd_ctx_device_bytes(fhd_ctx* c) { return c ? (unsigned long long)c->arena.bytes : 0ull; }

static int check_ptrs(fhd_ctx* ctx, const void* const* a, int n) {
    if (!ctx) return FHD_ERR_BAD_ARG;
    if (!a) return FHD_ERR_BAD_ARG;
    for (int i = 0; i < n; i++)
        if (!a[i]) return FHD_ERR_BAD_ARG;
    return 0;
}

static int nE_of(fhd_ctx* c) { return c->dim == 2 ? 1 : 3; }

static int finish(fhd_ctx* ctx, int rc) {
    if (rc < 0) return rc;
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        set_last_error(cudaGetErrorString(cudaGetLastError()));
        return FHD_ERR_CUDA;
    }
    if (int e = dev_err_check(ctx)) return e;
    return rc;
}

int fhd_dev_apply_matrix(fhd_ctx* ctx, double* const b_u[], double* b_p, const double* const x_u[],
                         const double* x_p, const double* const alpha_fc[], const double* beta,
                         const double* const beta_ed[], const double* gamma, double theta_alpha) {
    int rc = check_ptrs(ctx, (const void* const*)b_u, ctx ? ctx->dim : 0);
    if (!rc) rc = check_ptrs(ctx, (const void* const*)x_u, ctx->dim);
    if (!rc) rc = check_ptrs(ctx, (const void* const*)alpha_fc, ctx->dim);
    if (!rc) rc = check_ptrs(ctx, (const void* const*)beta_ed, nE_of(ctx));
    if (!rc && (!b_p || !x_p || !beta || !gamma)) rc = FHD_ERR_BAD_ARG;
    if (rc) return rc;
    for (int c = 0; c < 3; c++) ctx->alpha_fc[c] = c < ctx->dim ? alpha_fc[c] : nullptr;
    for (int e = 0; e < 3; e++) ctx->beta_ed[e] = e < nE_of(ctx) ? beta_ed[e] : nullptr;
    ctx->beta = beta;
    ctx->gamma = gamma;
    ctx->theta = theta_alpha;
    CSVec<double> x;
    SVec<double> o;
    for (int c = 0; c < 4; c++) { x.c[c] = nullptr; o.c[c] = nullptr; }
    for (int c = 0; c < ctx->dim; c++) { x.c[c] = x_u[c]; o.c[c] = b_u[c]; }
    x.c[ctx->dim] = x_p;
    o.c[ctx->dim] = b_p;
    return finish(ctx, stokes_apply(ctx, x, x, o, 0));
}

int fhd_dev_apply_precon(fhd_ctx* ctx, const double* const b_u[], const double* b_p, double* const x_u[],
                         double* x_p, const double* const alpha_fc[], const double* beta,
                         const double* const beta_ed[], const double* gamma, double theta_alpha) {
    int rc = check_ptrs(ctx, (const void* const*)b_u, ctx ? ctx->dim : 0);
    if (!rc) rc = check_ptrs(ctx, (const void* const*)x_u, ctx->dim);
    if (!rc) rc = check_ptrs(ctx, (const void* const*)alpha_fc, ctx->dim);
    if (!rc) rc = check_ptrs(ctx, (const void* const*)beta_ed, nE_of(ctx));
    if (!rc && (!b_p || !x_p || !beta || !gamma)) rc = FHD_ERR_BAD_ARG;
    if (rc) return rc;
    rc = prepare(ctx, alpha_fc, beta, beta_ed, gamma, theta_alpha);
    if (rc) return rc;
    CSVec<double> b;
    SVec<double> x;
    for (int c = 0; c < 4; c++) { b.c[c] = nullptr; x.c[c] = nullptr; }
    for (int c = 0; c < ctx->dim; c++) { b.c[c] = b_u[c]; x.c[c] = x_u[c]; }
    b.c[ctx->dim] = b_p;
    x.c[ctx->dim] = x_p;
    return finish(ctx, precon(ctx, b, x));
}

int fhd_dev_stag_mg_solver(fhd_ctx* ctx, const double* const alpha_fc[], const double* beta,
                           const double* const beta_ed[], const double* gamma, double theta_alpha,
                           double* const phi[], const double* const rhs[]) {
    int rc = check_ptrs(ctx, (const void* const*)phi, ctx ? ctx->dim : 0);
    if (!rc) rc = check_ptrs(ctx, (const void* const*)rhs, ctx->dim);
    if (!rc) rc = check_ptrs(ctx, (const void* const*)alpha_fc, ctx->dim);
    if (!rc) rc = check_ptrs(ctx, (const void* const*)beta_ed, nE_of(ctx));
    if (!rc && (!beta || !gamma)) rc = FHD_ERR_BAD_ARG;
    if (rc) return rc;
    rc = prepare(ctx, alpha_fc, beta, beta_ed, gamma, theta_alpha);
    if (rc) return rc;
    return finish(ctx, stag_mg_solve_dev(ctx, phi, rhs));
}

int fhd_dev_gmres(fhd_ctx* ctx, const double* const b_u[], const double* b_p, double* const x_u[], double* x_p,
                  const double* const alpha_fc[], const double* beta, const double* const beta_ed[],
                  const double* gamma, double theta_alpha, double* norm_pre_rhs, fhd_solve_stats* stats) {
    int rc = check_ptrs(ctx, (const void* const*)b_u, ctx ? ctx->dim : 0);
    if (!rc) rc = check_ptrs(ctx, (const void* const*)x_u, ctx->dim);
    if (!rc) rc = check_ptrs(ctx, (const void* const*)alpha_fc, ctx->dim);
    if (!rc) rc = check_ptrs(ctx, (const void* const*)beta_ed, nE_of(ctx));
    if (!rc && (!b_p || !x_p || !beta || !gamma)) rc = FHD_ERR_BAD_ARG;
    if (rc) return rc;
    // scale_factor (gmres.f90:118-135, 442-459): solve for scale*x_p with
    // theta_alpha, b_u and the viscosities scaled.  The reference scales the
    // caller's multifabs in place and unscales them on exit; here the scaled
    // operands are private stream-ordered copies, so the caller's b_u, beta,
    // gamma and beta_ed are not touched.  x_p is scaled in place and
    // unscaled by the reference's multiplication with 1/scale_factor.
    const double sf = ctx->p.scale_factor;
    if (!(sf > 0.0) && !(sf < 0.0)) {
        set_last_error("gmres: scale_factor must be non-zero");
        return FHD_ERR_BAD_ARG;
    }
    const int dim = ctx->dim, nE = nE_of(ctx);
    const i64 nc = ctx->g0.nc;
    cudaStream_t st = ctx->stream;
    const double* bu_s[3] = {b_u[0], dim > 1 ? b_u[1] : nullptr, dim > 2 ? b_u[2] : nullptr};
    const double* bed_s[3] = {beta_ed[0], nE > 1 ? beta_ed[1] : nullptr, nE > 2 ? beta_ed[2] : nullptr};
    const double *beta_s = beta, *gamma_s = gamma;
    double theta = theta_alpha;
    double* own = nullptr;
    const int nb = flat_blocks(nc);
    if (sf != 1.0) {
        FHD_CUDA_TRY(cudaMallocAsync((void**)&own, sizeof(double) * (size_t)nc * (dim + 2 + nE), st));
        int slot = 0;
        auto scaled = [&](const double* in) {
            double* o = own + (i64)(slot++) * nc;
            k_copy_conv<double, double><<<nb, 256, 0, st>>>(nc, o, in, sf);
            ctx->launches++;
            return (const double*)o;
        };
        theta = theta * sf;
        k_copy_conv<double, double><<<nb, 256, 0, st>>>(nc, x_p, x_p, sf);
        ctx->launches++;
        for (int c = 0; c < dim; c++) bu_s[c] = scaled(b_u[c]);
        beta_s = scaled(beta);
        gamma_s = scaled(gamma);
        for (int e = 0; e < nE; e++) bed_s[e] = scaled(beta_ed[e]);
        FHD_CUDA_TRY(cudaPeekAtLastError());
    }
    rc = prepare(ctx, alpha_fc, beta_s, bed_s, gamma_s, theta);
    CSVec<double> b;
    SVec<double> x;
    for (int c = 0; c < 4; c++) { b.c[c] = nullptr; x.c[c] = nullptr; }
    for (int c = 0; c < dim; c++) { b.c[c] = bu_s[c]; x.c[c] = x_u[c]; }
    b.c[dim] = b_p;
    x.c[dim] = x_p;
    if (!rc) rc = gmres_dev(ctx, b, x, norm_pre_rhs, stats);
    if (sf != 1.0) {
        if (rc >= 0) {
            k_copy_conv<double, double><<<nb, 256, 0, st>>>(nc, x_p, x_p, 1.0 / sf);
            ctx->launches++;
        }
        cudaFreeAsync(own, st);
    }
    return finish(ctx, rc);
}

}  // extern "C"
