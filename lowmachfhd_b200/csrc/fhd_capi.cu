// fhd_capi.cu -- the host BoxLib-fab entry points (the drop-in boundary a
// Fortran driver binds through iso_c_binding).
//
// A fab is a Fortran column-major array (lo-ng : hi+nodal+ng, ..., ncomp)
// holding one box of a multifab.  Inputs are copied to the device and
// gathered into the canonical periodic layout (each box contributes its
// cells lo..hi in every direction, so the duplicated periodic face hi+1 is
// taken from the box that owns it as face lo, as multifab_internal_sync
// keeps them equal).  Outputs are scattered back over the whole fab,
// ghost cells included, which is the periodic multifab_fill_boundary.
#include <cstring>

#include "fhd_solver.cuh"

namespace fhd {

struct FabDesc {
    int lo[3], hi[3], nodal[3], ng;
    int ext[3];  // extents incl. ghosts
};

static FabDesc desc_of(const fhd_fab& f, int dim) {
    FabDesc d;
    for (int k = 0; k < 3; k++) {
        const bool act = k < dim;
        d.lo[k] = act ? f.lo[k] : 0;
        d.hi[k] = act ? f.hi[k] : 0;
        d.nodal[k] = act ? (f.nodal[k] ? 1 : 0) : 0;
    }
    d.ng = f.ng;
    for (int k = 0; k < 3; k++) d.ext[k] = (k < dim) ? d.hi[k] - d.lo[k] + 1 + d.nodal[k] + 2 * d.ng : 1;
    return d;
}

static i64 fab_elems(const FabDesc& d) { return (i64)d.ext[0] * d.ext[1] * d.ext[2]; }

// fab -> canonical over the box's valid cells lo..hi
__global__ void k_gather(Grid g, FabDesc d, const double* __restrict__ fab, double* out) {
    const int bx = d.hi[0] - d.lo[0] + 1, by = d.hi[1] - d.lo[1] + 1, bz = d.hi[2] - d.lo[2] + 1;
    const i64 n = (i64)bx * by * bz;
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n; t += (i64)gridDim.x * blockDim.x) {
        const int a = (int)(t % bx), b = (int)((t / bx) % by), c = (int)(t / ((i64)bx * by));
        const int i = d.lo[0] + a, j = d.lo[1] + b, k = d.lo[2] + c;
        const i64 src = (i64)(a + d.ng) + (i64)d.ext[0] * ((i64)(b + (g.dim > 1 ? d.ng : 0)) +
                                                             (i64)d.ext[1] * (i64)(c + (g.dim > 2 ? d.ng : 0)));
        const i64 dst = (i64)wrapc(i, g.n[0]) + (i64)g.n[0] * ((i64)wrapc(j, g.n[1]) + (i64)g.n[1] * wrapc(k, g.n[2]));
        out[dst] = fab[src];
    }
}

// One whole-domain fab -> the wall-extended layout of an edge set: the
// cells lo..hi, plus the nodal plane hi+1 in the directions with xt[d] = 1
// (a wall direction in which the fab is nodal: the high wall's edges, which
// the reference draws independently).  Extents m[d] = n[d] + xt[d].
struct EdgeGather {
    int xt[3], m[3];
};
__global__ void k_gather_ext(FabDesc d, EdgeGather X, int dim, const double* __restrict__ fab, double* out) {
    const int bx = X.m[0], by = X.m[1], bz = X.m[2];
    const i64 n = (i64)bx * by * bz;
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n; t += (i64)gridDim.x * blockDim.x) {
        const int a = (int)(t % bx), b = (int)((t / bx) % by), c = (int)(t / ((i64)bx * by));
        const i64 src = (i64)(a + d.ng) + (i64)d.ext[0] * ((i64)(b + (dim > 1 ? d.ng : 0)) +
                                                             (i64)d.ext[1] * (i64)(c + (dim > 2 ? d.ng : 0)));
        out[t] = fab[src];
    }
}

// canonical -> whole fab (valid, nodal duplicate and ghosts)
__global__ void k_scatter(Grid g, FabDesc d, const double* __restrict__ in, double* fab) {
    const i64 n = (i64)d.ext[0] * d.ext[1] * d.ext[2];
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n; t += (i64)gridDim.x * blockDim.x) {
        const int a = (int)(t % d.ext[0]), b = (int)((t / d.ext[0]) % d.ext[1]), c = (int)(t / ((i64)d.ext[0] * d.ext[1]));
        const int i = d.lo[0] - d.ng + a;
        const int j = (g.dim > 1) ? d.lo[1] - d.ng + b : 0;
        const int k = (g.dim > 2) ? d.lo[2] - d.ng + c : 0;
        const int ii = ((i % g.n[0]) + g.n[0]) % g.n[0];
        const int jj = ((j % g.n[1]) + g.n[1]) % g.n[1];
        const int kk = ((k % g.n[2]) + g.n[2]) % g.n[2];
        fab[t] = in[(i64)ii + (i64)g.n[0] * ((i64)jj + (i64)g.n[1] * kk)];
    }
}

struct HostPath {
    bool ready = false;
    double* arr[24] = {nullptr};  // canonical device copies of the operands
    double* stage = nullptr;      // raw fab staging
    i64 stage_elems = 0;
};

static int ensure_stage(fhd_ctx* ctx, HostPath& H, i64 elems) {
    if (elems <= H.stage_elems) return 0;
    if (H.stage) cudaFree(H.stage);
    H.stage = nullptr;
    H.stage_elems = 0;
    FHD_CUDA_TRY(cudaMalloc(&H.stage, sizeof(double) * (size_t)elems));
    H.stage_elems = elems;
    return 0;
}

// per-context host-path state
static HostPath& host_path(fhd_ctx* ctx);

static int check_mf(fhd_ctx* ctx, const fhd_multifab* mf, int want_ng) {
    if (!mf || mf->nfabs < 1 || !mf->fabs) return FHD_ERR_BAD_ARG;
    for (int b = 0; b < mf->nfabs; b++) {
        const fhd_fab& f = mf->fabs[b];
        if (!f.data || f.ng < 0 || f.ncomp < 1) return FHD_ERR_BAD_ARG;
        if (f.ng < want_ng) return FHD_ERR_BAD_GHOSTS;
        for (int d = 0; d < ctx->dim; d++)
            if (f.lo[d] < 0 || f.hi[d] >= ctx->n[d] || f.hi[d] < f.lo[d]) return FHD_ERR_BAD_ARG;
    }
    return 0;
}

int mf_to_dev(fhd_ctx* ctx, const fhd_multifab* mf, double* dst) {
    HostPath& H = host_path(ctx);
    for (int b = 0; b < mf->nfabs; b++) {
        const fhd_fab& f = mf->fabs[b];
        FabDesc d = desc_of(f, ctx->dim);
        const i64 ne = fab_elems(d);
        int rc = ensure_stage(ctx, H, ne);
        if (rc) return rc;
        FHD_CUDA_TRY(cudaMemcpyAsync(H.stage, f.data, sizeof(double) * ne, cudaMemcpyHostToDevice, ctx->stream));
        k_gather<<<flat_blocks(ne), 256, 0, ctx->stream>>>(ctx->g0, d, H.stage, dst);
        ctx->launches++;
        FHD_CUDA_TRY(cudaPeekAtLastError());
    }
    return 0;
}

// an edge multifab of set e (2D the nodes; 3D xy, xz, yz) in a context with
// walls -> the wall-extended layout; the multifab must be one whole-domain
// fab, nodal exactly in the set's directions
static int mf_to_dev_edge(fhd_ctx* ctx, const fhd_multifab* mf, int e, double* dst) {
    const int dim = ctx->dim;
    const int da = (dim == 3 && e == 2) ? 1 : 0, db = (dim == 3 && e != 0) ? 2 : 1;
    if (mf->nfabs != 1) {
        set_last_error("edge multifab with walls: one whole-domain fab expected");
        return FHD_ERR_BAD_ARG;
    }
    const fhd_fab& f = mf->fabs[0];
    FabDesc d = desc_of(f, dim);
    EdgeGather X;
    for (int k = 0; k < 3; k++) {
        const bool in_set = k < dim && (k == da || k == db);
        if (k < dim && (d.lo[k] != 0 || d.hi[k] != ctx->n[k] - 1 || d.nodal[k] != (in_set ? 1 : 0))) {
            set_last_error("edge multifab with walls: one whole-domain fab, nodal in the edge set's directions");
            return FHD_ERR_BAD_ARG;
        }
        X.xt[k] = in_set && ctx->walls.lo[k] != 0 ? 1 : 0;
        X.m[k] = (k < dim ? ctx->n[k] : 1) + X.xt[k];
    }
    HostPath& H = host_path(ctx);
    const i64 ne = fab_elems(d);
    if (int rc = ensure_stage(ctx, H, ne)) return rc;
    FHD_CUDA_TRY(cudaMemcpyAsync(H.stage, f.data, sizeof(double) * ne, cudaMemcpyHostToDevice, ctx->stream));
    k_gather_ext<<<flat_blocks((i64)X.m[0] * X.m[1] * X.m[2]), 256, 0, ctx->stream>>>(d, X, dim, H.stage, dst);
    ctx->launches++;
    FHD_CUDA_TRY(cudaPeekAtLastError());
    return 0;
}

int dev_to_mf(fhd_ctx* ctx, const double* src, const fhd_multifab* mf) {
    HostPath& H = host_path(ctx);
    for (int b = 0; b < mf->nfabs; b++) {
        const fhd_fab& f = mf->fabs[b];
        FabDesc d = desc_of(f, ctx->dim);
        const i64 ne = fab_elems(d);
        int rc = ensure_stage(ctx, H, ne);
        if (rc) return rc;
        k_scatter<<<flat_blocks(ne), 256, 0, ctx->stream>>>(ctx->g0, d, src, H.stage);
        ctx->launches++;
        FHD_CUDA_TRY(cudaPeekAtLastError());
        FHD_CUDA_TRY(cudaMemcpyAsync(f.data, H.stage, sizeof(double) * ne, cudaMemcpyDeviceToHost, ctx->stream));
        // the staging buffer is reused by the next box
        FHD_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    }
    return 0;
}

}  // namespace fhd

using namespace fhd;

// host-path state lives beside the context, keyed by its address
#include <map>
#include <mutex>
static std::mutex g_hp_mu;
static std::map<fhd_ctx*, HostPath*> g_hp;

namespace fhd {
static HostPath& host_path(fhd_ctx* ctx) {
    std::lock_guard<std::mutex> lk(g_hp_mu);
    auto it = g_hp.find(ctx);
    if (it != g_hp.end()) return *it->second;
    HostPath* h = new HostPath();
    g_hp[ctx] = h;
    return *h;
}
}  // namespace fhd

extern "C" void fhd_host_path_release(fhd_ctx* ctx) {
    std::lock_guard<std::mutex> lk(g_hp_mu);
    auto it = g_hp.find(ctx);
    if (it == g_hp.end()) return;
    HostPath* h = it->second;
    if (h->stage) cudaFree(h->stage);
    for (double* a : h->arr)
        if (a) cudaFree(a);
    delete h;
    g_hp.erase(it);
}

namespace {

enum { A_BU = 0, A_BP = 3, A_XU = 4, A_XP = 7, A_AL = 8, A_BE = 11, A_BED = 12, A_GA = 15, A_COUNT = 16 };

int host_arrays(fhd_ctx* ctx, HostPath*& out) {
    HostPath& H = host_path(ctx);
    if (!H.ready) {
        for (int i = 0; i < A_COUNT; i++) {
            FHD_CUDA_TRY(cudaMalloc(&H.arr[i], sizeof(double) * (size_t)ctx->g0.nc));
        }
        H.ready = true;
    }
    out = &H;
    return 0;
}

struct Operands {
    double* b_u[3];
    double* b_p;
    double* x_u[3];
    double* x_p;
    double* al[3];
    double* be;
    double* bed[3];
    double* ga;
};

int load_coeffs(fhd_ctx* ctx, HostPath* H, Operands& o, const fhd_multifab* alpha_fc, const fhd_multifab* beta,
                const fhd_multifab* beta_ed, const fhd_multifab* gamma) {
    const int dim = ctx->dim, nE = dim == 2 ? 1 : 3;
    for (int c = 0; c < 3; c++) {
        o.b_u[c] = H->arr[A_BU + c];
        o.x_u[c] = H->arr[A_XU + c];
        o.al[c] = H->arr[A_AL + c];
        o.bed[c] = H->arr[A_BED + c];
    }
    o.b_p = H->arr[A_BP];
    o.x_p = H->arr[A_XP];
    o.be = H->arr[A_BE];
    o.ga = H->arr[A_GA];
    int rc;
    for (int c = 0; c < dim; c++) {
        if ((rc = check_mf(ctx, &alpha_fc[c], 0))) return rc;
        if ((rc = mf_to_dev(ctx, &alpha_fc[c], o.al[c]))) return rc;
    }
    for (int e = 0; e < nE; e++) {
        if ((rc = check_mf(ctx, &beta_ed[e], 0))) return rc;
        if ((rc = mf_to_dev(ctx, &beta_ed[e], o.bed[e]))) return rc;
    }
    if ((rc = check_mf(ctx, beta, 0)) || (rc = check_mf(ctx, gamma, 0))) return rc;
    if ((rc = mf_to_dev(ctx, beta, o.be))) return rc;
    if ((rc = mf_to_dev(ctx, gamma, o.ga))) return rc;
    return 0;
}

// one component of a multi-component multifab, as a one-component view
// (the data pointer of each fab advanced by comp whole components)
void comp_view(const fhd_multifab& mf, int dim, int comp, std::vector<fhd_fab>& store, fhd_multifab& out) {
    store.assign(mf.fabs, mf.fabs + mf.nfabs);
    for (auto& f : store) {
        FabDesc d = desc_of(f, dim);
        f.data = f.data + (i64)comp * fab_elems(d);
    }
    out.nfabs = mf.nfabs;
    out.fabs = store.data();
}

int check_ncomp(const fhd_multifab& mf, int want) {
    for (int b = 0; b < mf.nfabs; b++)
        if (mf.fabs[b].ncomp < want) return FHD_ERR_BAD_ARG;
    return 0;
}

// every component of a multifab to its own canonical device array
int mf_comps_to_dev(fhd_ctx* ctx, const fhd_multifab& mf, int ncomp, double* const dst[]) {
    std::vector<fhd_fab> store;
    fhd_multifab one;
    for (int c = 0; c < ncomp; c++) {
        comp_view(mf, ctx->dim, c, store, one);
        if (int rc = mf_to_dev(ctx, &one, dst[c])) return rc;
        // the view's fab descriptors live in store until the copies are queued
        FHD_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    }
    return 0;
}

int dev_to_mf_comps(fhd_ctx* ctx, const double* const src[], int ncomp, const fhd_multifab& mf) {
    std::vector<fhd_fab> store;
    fhd_multifab one;
    for (int c = 0; c < ncomp; c++) {
        comp_view(mf, ctx->dim, c, store, one);
        if (int rc = dev_to_mf(ctx, src[c], &one)) return rc;
    }
    return 0;
}

// per-call device arrays of nc doubles, freed on scope exit
struct DevArrays {
    std::vector<double*> a;
    int alloc(int n, i64 nc) {
        a.assign(n, nullptr);
        for (int i = 0; i < n; i++)
            if (cudaMalloc(&a[i], sizeof(double) * (size_t)nc) != cudaSuccess) return FHD_ERR_OOM;
        return 0;
    }
    ~DevArrays() {
        for (double* p : a)
            if (p) cudaFree(p);
    }
};

}  // namespace

extern "C" {

int fhd_gmres(fhd_ctx* ctx, const fhd_multifab* b_u, const fhd_multifab* b_p, const fhd_multifab* x_u,
              const fhd_multifab* x_p, const fhd_multifab* alpha_fc, const fhd_multifab* beta,
              const fhd_multifab* beta_ed, const fhd_multifab* gamma, double* theta_alpha, double* norm_pre_rhs,
              fhd_solve_stats* stats) {
    if (!ctx || !b_u || !b_p || !x_u || !x_p || !alpha_fc || !beta || !beta_ed || !gamma || !theta_alpha)
        return FHD_ERR_BAD_ARG;
    const int dim = ctx->dim;
    int rc;
    // x needs gmres_spatial_order / 2 ghost cells (apply_matrix.f90:54-67)
    const int xg = ctx->p.gmres_spatial_order == 4 ? 2 : 1;
    for (int c = 0; c < dim; c++)
        if ((rc = check_mf(ctx, &x_u[c], xg)) || (rc = check_mf(ctx, &b_u[c], 0))) return rc;
    if ((rc = check_mf(ctx, x_p, xg)) || (rc = check_mf(ctx, b_p, 0))) return rc;
    HostPath* H;
    if ((rc = host_arrays(ctx, H))) return rc;
    Operands o;
    if ((rc = load_coeffs(ctx, H, o, alpha_fc, beta, beta_ed, gamma))) return rc;
    for (int c = 0; c < dim; c++) {
        if ((rc = mf_to_dev(ctx, &b_u[c], o.b_u[c]))) return rc;
        if ((rc = mf_to_dev(ctx, &x_u[c], o.x_u[c]))) return rc;
    }
    if ((rc = mf_to_dev(ctx, b_p, o.b_p)) || (rc = mf_to_dev(ctx, x_p, o.x_p))) return rc;
    const double* cb[3] = {o.b_u[0], o.b_u[1], o.b_u[2]};
    const double* ca[3] = {o.al[0], o.al[1], o.al[2]};
    const double* ce[3] = {o.bed[0], o.bed[1], o.bed[2]};
    int st = fhd_dev_gmres(ctx, cb, o.b_p, o.x_u, o.x_p, ca, o.be, ce, o.ga, *theta_alpha, norm_pre_rhs, stats);
    if (st < 0) return st;
    for (int c = 0; c < dim; c++)
        if ((rc = dev_to_mf(ctx, o.x_u[c], &x_u[c]))) return rc;
    if ((rc = dev_to_mf(ctx, o.x_p, x_p))) return rc;
    return st;
}

int fhd_apply_precon(fhd_ctx* ctx, const fhd_multifab* b_u, const fhd_multifab* b_p, const fhd_multifab* x_u,
                     const fhd_multifab* x_p, const fhd_multifab* alpha_fc, const fhd_multifab* beta,
                     const fhd_multifab* beta_ed, const fhd_multifab* gamma, double theta_alpha) {
    if (!ctx || !b_u || !b_p || !x_u || !x_p || !alpha_fc || !beta || !beta_ed || !gamma) return FHD_ERR_BAD_ARG;
    const int dim = ctx->dim;
    int rc;
    for (int c = 0; c < dim; c++)
        if ((rc = check_mf(ctx, &x_u[c], 0)) || (rc = check_mf(ctx, &b_u[c], 0))) return rc;
    if ((rc = check_mf(ctx, x_p, 0)) || (rc = check_mf(ctx, b_p, 0))) return rc;
    HostPath* H;
    if ((rc = host_arrays(ctx, H))) return rc;
    Operands o;
    if ((rc = load_coeffs(ctx, H, o, alpha_fc, beta, beta_ed, gamma))) return rc;
    for (int c = 0; c < dim; c++)
        if ((rc = mf_to_dev(ctx, &b_u[c], o.b_u[c]))) return rc;
    if ((rc = mf_to_dev(ctx, b_p, o.b_p))) return rc;
    const double* cb[3] = {o.b_u[0], o.b_u[1], o.b_u[2]};
    const double* ca[3] = {o.al[0], o.al[1], o.al[2]};
    const double* ce[3] = {o.bed[0], o.bed[1], o.bed[2]};
    rc = fhd_dev_apply_precon(ctx, cb, o.b_p, o.x_u, o.x_p, ca, o.be, ce, o.ga, theta_alpha);
    if (rc < 0) return rc;
    for (int c = 0; c < dim; c++)
        if ((rc = dev_to_mf(ctx, o.x_u[c], &x_u[c]))) return rc;
    return dev_to_mf(ctx, o.x_p, x_p);
}

int fhd_apply_matrix(fhd_ctx* ctx, const fhd_multifab* b_u, const fhd_multifab* b_p, const fhd_multifab* x_u,
                     const fhd_multifab* x_p, const fhd_multifab* alpha_fc, const fhd_multifab* beta,
                     const fhd_multifab* beta_ed, const fhd_multifab* gamma, double theta_alpha) {
    if (!ctx || !b_u || !b_p || !x_u || !x_p || !alpha_fc || !beta || !beta_ed || !gamma) return FHD_ERR_BAD_ARG;
    const int dim = ctx->dim;
    int rc;
    // x needs gmres_spatial_order / 2 ghost cells (apply_matrix.f90:54-67)
    const int xg = ctx->p.gmres_spatial_order == 4 ? 2 : 1;
    for (int c = 0; c < dim; c++)
        if ((rc = check_mf(ctx, &x_u[c], xg)) || (rc = check_mf(ctx, &b_u[c], 0))) return rc;
    if ((rc = check_mf(ctx, x_p, xg)) || (rc = check_mf(ctx, b_p, 0))) return rc;
    HostPath* H;
    if ((rc = host_arrays(ctx, H))) return rc;
    Operands o;
    if ((rc = load_coeffs(ctx, H, o, alpha_fc, beta, beta_ed, gamma))) return rc;
    for (int c = 0; c < dim; c++)
        if ((rc = mf_to_dev(ctx, &x_u[c], o.x_u[c]))) return rc;
    if ((rc = mf_to_dev(ctx, x_p, o.x_p))) return rc;
    const double* cx[3] = {o.x_u[0], o.x_u[1], o.x_u[2]};
    const double* ca[3] = {o.al[0], o.al[1], o.al[2]};
    const double* ce[3] = {o.bed[0], o.bed[1], o.bed[2]};
    rc = fhd_dev_apply_matrix(ctx, o.b_u, o.b_p, cx, o.x_p, ca, o.be, ce, o.ga, theta_alpha);
    if (rc < 0) return rc;
    for (int c = 0; c < dim; c++)
        if ((rc = dev_to_mf(ctx, o.b_u[c], &b_u[c]))) return rc;
    return dev_to_mf(ctx, o.b_p, b_p);
}

int fhd_stochastic_m_fluxdiv(fhd_ctx* ctx, const fhd_stoch_params* sp, const fhd_multifab* stoch_m_force,
                             int increment, const fhd_multifab* eta, const fhd_multifab* eta_ed,
                             const fhd_multifab* temperature, const fhd_multifab* temperature_ed, double dt,
                             const double* weights, int n_rngs, const fhd_multifab* W_cc, const fhd_multifab* W_ed) {
    if (!ctx || !sp || !stoch_m_force || !eta || !eta_ed || !temperature || !temperature_ed || !weights || !W_cc ||
        !W_ed || n_rngs < 1 || n_rngs > 4)
        return FHD_ERR_BAD_ARG;
    const int dim = ctx->dim, nE = dim == 2 ? 1 : 3;
    const i64 nc = ctx->g0.nc;
    // per-call device arrays: force (dim), eta, T, eta_ed, T_ed (nE each),
    // and the component-split random fields
    const int ncc = n_rngs * dim, ned = n_rngs * 2 * nE;
    const int total = dim + 2 + 2 * nE + ncc + ned;
    // with walls an edge set that contains a wall direction has the high
    // wall's plane too (the device entry's wall-extended layout)
    i64 ne[3] = {nc, nc, nc};
    if (ctx->has_walls)
        for (int e = 0; e < nE; e++) {
            const int da = (dim == 3 && e == 2) ? 1 : 0, db = (dim == 3 && e != 0) ? 2 : 1;
            ne[e] = 1;
            for (int k = 0; k < dim; k++) ne[e] *= ctx->n[k] + ((k == da || k == db) && ctx->walls.lo[k] != 0 ? 1 : 0);
        }
    auto elems_of = [&](int i) -> i64 {
        if (i >= dim + 2 && i < dim + 2 + 2 * nE) return ne[(i - dim - 2) % nE];  // eta_ed, T_ed
        if (i >= dim + 2 + 2 * nE + ncc) return ne[((i - dim - 2 - 2 * nE - ncc) / 2) % nE];  // W_ed
        return nc;
    };
    std::vector<double*> A(total, nullptr);
    int rc = 0;
    for (int i = 0; i < total && !rc; i++)
        if (cudaMalloc(&A[i], sizeof(double) * elems_of(i)) != cudaSuccess) rc = FHD_ERR_OOM;
    auto cleanup = [&]() {
        for (double* p : A)
            if (p) cudaFree(p);
    };
    if (rc) { cleanup(); return rc; }
    double* force[3] = {A[0], A[1], dim == 3 ? A[2] : nullptr};
    double* d_eta = A[dim];
    double* d_T = A[dim + 1];
    double* d_eed[3] = {nullptr, nullptr, nullptr};
    double* d_Ted[3] = {nullptr, nullptr, nullptr};
    for (int e = 0; e < nE; e++) {
        d_eed[e] = A[dim + 2 + e];
        d_Ted[e] = A[dim + 2 + nE + e];
    }
    double** d_Wcc = &A[dim + 2 + 2 * nE];
    double** d_Wed = &A[dim + 2 + 2 * nE + ncc];
    // multi-component fabs are split per component by offsetting the data
    auto comp_mf = [&](const fhd_multifab& mf, int comp, std::vector<fhd_fab>& store, fhd_multifab& out) {
        store.assign(mf.fabs, mf.fabs + mf.nfabs);
        for (auto& f : store) {
            FabDesc d = desc_of(f, dim);
            f.data = f.data + (i64)comp * fab_elems(d);
        }
        out.nfabs = mf.nfabs;
        out.fabs = store.data();
    };
    do {
        for (int c = 0; c < dim && !rc; c++)
            if ((rc = check_mf(ctx, &stoch_m_force[c], 0)) == 0 && increment) rc = mf_to_dev(ctx, &stoch_m_force[c], force[c]);
        if (rc) break;
        if ((rc = check_mf(ctx, eta, 0)) || (rc = mf_to_dev(ctx, eta, d_eta))) break;
        if ((rc = check_mf(ctx, temperature, 0)) || (rc = mf_to_dev(ctx, temperature, d_T))) break;
        // an edge multifab: the periodic gather, or with walls the extended one
        auto edge_to_dev = [&](const fhd_multifab* mf, int e, double* dst) {
            return ctx->has_walls ? mf_to_dev_edge(ctx, mf, e, dst) : mf_to_dev(ctx, mf, dst);
        };
        for (int e = 0; e < nE && !rc; e++) {
            if ((rc = check_mf(ctx, &eta_ed[e], 0)) || (rc = edge_to_dev(&eta_ed[e], e, d_eed[e]))) break;
            if ((rc = check_mf(ctx, &temperature_ed[e], 0)) || (rc = edge_to_dev(&temperature_ed[e], e, d_Ted[e])))
                break;
        }
        if (rc) break;
        std::vector<fhd_fab> store;
        fhd_multifab one;
        for (int r = 0; r < n_rngs && !rc; r++) {
            for (int c = 0; c < dim && !rc; c++) {
                if ((rc = check_mf(ctx, &W_cc[r], 0))) break;
                for (int b = 0; b < W_cc[r].nfabs; b++)
                    if (W_cc[r].fabs[b].ncomp < dim) rc = FHD_ERR_BAD_ARG;
                if (rc) break;
                comp_mf(W_cc[r], c, store, one);
                rc = mf_to_dev(ctx, &one, d_Wcc[r * dim + c]);
                if (!rc) rc = cudaStreamSynchronize(ctx->stream) == cudaSuccess ? 0 : FHD_ERR_CUDA;
            }
            for (int e = 0; e < nE && !rc; e++) {
                if ((rc = check_mf(ctx, &W_ed[r * nE + e], 0))) break;
                for (int b = 0; b < W_ed[r * nE + e].nfabs; b++)
                    if (W_ed[r * nE + e].fabs[b].ncomp < 2) rc = FHD_ERR_BAD_ARG;
                if (rc) break;
                for (int comp = 0; comp < 2 && !rc; comp++) {
                    comp_mf(W_ed[r * nE + e], comp, store, one);
                    rc = edge_to_dev(&one, e, d_Wed[r * 2 * nE + 2 * e + comp]);
                    if (!rc) rc = cudaStreamSynchronize(ctx->stream) == cudaSuccess ? 0 : FHD_ERR_CUDA;
                }
            }
        }
        if (rc) break;
        const double* ceed[3] = {d_eed[0], d_eed[1], d_eed[2]};
        const double* cTed[3] = {d_Ted[0], d_Ted[1], d_Ted[2]};
        std::vector<const double*> cWcc(d_Wcc, d_Wcc + ncc), cWed(d_Wed, d_Wed + ned);
        rc = fhd_dev_stochastic_m_fluxdiv(ctx, sp, force, increment, d_eta, ceed, d_T, cTed, dt, weights, n_rngs,
                                          cWcc.data(), cWed.data());
        if (rc) break;
        for (int c = 0; c < dim && !rc; c++) rc = dev_to_mf(ctx, force[c], &stoch_m_force[c]);
    } while (0);
    cudaStreamSynchronize(ctx->stream);
    cleanup();
    return rc;
}

int fhd_stag_mg_solve(fhd_ctx* ctx, const fhd_multifab* alpha_fc, const fhd_multifab* beta_cc,
                      const fhd_multifab* beta_ed, const fhd_multifab* gamma_cc, double theta_alpha,
                      const fhd_multifab* phi_fc, const fhd_multifab* rhs_fc) {
    if (!ctx || !alpha_fc || !beta_cc || !beta_ed || !gamma_cc || !phi_fc || !rhs_fc) return FHD_ERR_BAD_ARG;
    const int dim = ctx->dim;
    int rc;
    for (int c = 0; c < dim; c++)
        if ((rc = check_mf(ctx, &phi_fc[c], 1)) || (rc = check_mf(ctx, &rhs_fc[c], 0))) return rc;
    HostPath* H;
    if ((rc = host_arrays(ctx, H))) return rc;
    Operands o;
    if ((rc = load_coeffs(ctx, H, o, alpha_fc, beta_cc, beta_ed, gamma_cc))) return rc;
    for (int c = 0; c < dim; c++) {
        if ((rc = mf_to_dev(ctx, &rhs_fc[c], o.b_u[c]))) return rc;
        if ((rc = mf_to_dev(ctx, &phi_fc[c], o.x_u[c]))) return rc;
    }
    const double* cr[3] = {o.b_u[0], o.b_u[1], o.b_u[2]};
    const double* ca[3] = {o.al[0], o.al[1], o.al[2]};
    const double* ce[3] = {o.bed[0], o.bed[1], o.bed[2]};
    rc = fhd_dev_stag_mg_solver(ctx, ca, o.be, ce, o.ga, theta_alpha, o.x_u, cr);
    if (rc < 0) return rc;
    for (int c = 0; c < dim; c++)
        if (int r2 = dev_to_mf(ctx, o.x_u[c], &phi_fc[c])) return r2;
    return rc;
}

// walls: the high wall face of direction d is the fab's nodal plane hi+1,
// which the periodic scatter fills from face 0; write the wall's own factors
// (sqrtL_high_wall_plane) there.  One whole-domain fab, nodal in d; in the
// other directions its ghost positions wrap where periodic and clamp at a
// wall.
static int put_sqrtL_high_wall(fhd_ctx* ctx, const fhd_mixture_params* mp, const fhd_stoch_params* sp,
                               const double* const rho[], int d, int ncomp, const fhd_multifab& mf) {
    const int dim = ctx->dim;
    if (mf.nfabs != 1) {
        set_last_error("compute_sqrtLonsager_fc with walls: one whole-domain fab per direction expected");
        return FHD_ERR_BAD_ARG;
    }
    const fhd_fab& f = mf.fabs[0];
    const FabDesc fd = desc_of(f, dim);
    for (int k = 0; k < dim; k++)
        if (fd.lo[k] != 0 || fd.hi[k] != ctx->n[k] - 1 || fd.nodal[k] != (k == d ? 1 : 0)) {
            set_last_error("compute_sqrtLonsager_fc with walls: one whole-domain face fab per direction expected");
            return FHD_ERR_BAD_ARG;
        }
    const int u = d == 0 ? 1 : 0, v = d == 2 ? 1 : 2;
    const i64 nu = ctx->n[u], nv = v < dim ? ctx->n[v] : 1, np = nu * nv;
    DevArrays P;
    if (int rc = P.alloc(ncomp, np)) return rc;
    if (int rc = sqrtL_high_wall_plane(ctx, mp, sp, rho, d, P.a.data())) return rc;
    std::vector<double> h((size_t)np);
    const i64 ne = fab_elems(fd);
    for (int q = 0; q < ncomp; q++) {
        FHD_CUDA_TRY(cudaMemcpy(h.data(), P.a[q], sizeof(double) * np, cudaMemcpyDeviceToHost));
        double* base = f.data + (i64)q * ne;
        auto pos = [&](int k, int e) {  // fab offset e along direction k -> cell index
            const int c = e - fd.ng;
            if (ctx->walls.lo[k] == 0) return ((c % ctx->n[k]) + ctx->n[k]) % ctx->n[k];
            return c < 0 ? 0 : (c >= ctx->n[k] ? ctx->n[k] - 1 : c);
        };
        const int eu = fd.ext[u], ev = v < dim ? fd.ext[v] : 1;
        for (int b = 0; b < ev; b++)
            for (int a = 0; a < eu; a++) {
                int o[3] = {0, 0, 0};
                o[d] = fd.ng + ctx->n[d];  // the nodal plane hi+1
                o[u] = a;
                if (v < dim) o[v] = b;
                const i64 src = (i64)pos(u, a) + nu * (v < dim ? (i64)pos(v, b) : 0);
                base[(i64)o[0] + (i64)fd.ext[0] * ((i64)o[1] + (i64)fd.ext[1] * o[2])] = h[(size_t)src];
            }
    }
    return 0;
}

int fhd_compute_sqrtLonsager_fc(fhd_ctx* ctx, const fhd_mixture_params* mp, const fhd_stoch_params* sp,
                                const fhd_multifab* rho, const fhd_multifab* rhotot,
                                const fhd_multifab* sqrtLonsager_fc) {
    if (!ctx || !mp || !sp || !rho || !sqrtLonsager_fc) return FHD_ERR_BAD_ARG;
    if (int r0 = fhd::refuse_reservoirs(ctx, "fhd_compute_sqrtLonsager_fc")) return r0;
    if (mp->nspecies < 2 || mp->nspecies > 5) return FHD_ERR_UNSUPPORTED;
    const int dim = ctx->dim, ns = mp->nspecies;
    int rc;
    // rho is read on both sides of every face: one ghost cell
    if ((rc = check_mf(ctx, rho, 1)) || (rc = check_ncomp(*rho, ns))) return rc;
    if (rhotot && (rc = check_mf(ctx, rhotot, 0))) return rc;
    for (int d = 0; d < dim; d++)
        if ((rc = check_mf(ctx, &sqrtLonsager_fc[d], 0)) || (rc = check_ncomp(sqrtLonsager_fc[d], ns * ns))) return rc;
    DevArrays A;
    if ((rc = A.alloc(ns + dim * ns * ns, ctx->g0.nc))) return rc;
    double** d_rho = A.a.data();
    double** d_L = A.a.data() + ns;
    if ((rc = mf_comps_to_dev(ctx, *rho, ns, d_rho))) return rc;
    std::vector<const double*> crho(d_rho, d_rho + ns);
    if ((rc = fhd_dev_compute_sqrtLonsager_fc(ctx, mp, sp, crho.data(), d_L))) return rc;
    for (int d = 0; d < dim; d++) {
        std::vector<const double*> src(d_L + d * ns * ns, d_L + (d + 1) * ns * ns);
        if ((rc = dev_to_mf_comps(ctx, src.data(), ns * ns, sqrtLonsager_fc[d]))) return rc;
        if (ctx->has_walls && ctx->walls.lo[d] != 0 &&
            (rc = put_sqrtL_high_wall(ctx, mp, sp, crho.data(), d, ns * ns, sqrtLonsager_fc[d])))
            return rc;
    }
    return 0;
}

int fhd_stochastic_mass_fluxdiv(fhd_ctx* ctx, const fhd_mixture_params* mp, const fhd_stoch_params* sp,
                                const fhd_multifab* rho, const fhd_multifab* rhotot,
                                const fhd_multifab* sqrtLonsager_fc, const fhd_multifab* stoch_mass_fluxdiv,
                                const fhd_multifab* stoch_mass_flux, double dt, const double* weights, int n_rngs,
                                const fhd_multifab* W_fc, int increment) {
    if (!ctx || !mp || !sp || !sqrtLonsager_fc || !stoch_mass_fluxdiv || !weights || !W_fc || !(dt > 0.0))
        return FHD_ERR_BAD_ARG;
    if (int r0 = fhd::refuse_reservoirs(ctx, "fhd_stochastic_mass_fluxdiv")) return r0;
    if (mp->nspecies < 2 || mp->nspecies > 5 || n_rngs < 1 || n_rngs > 4) return FHD_ERR_UNSUPPORTED;
    const int dim = ctx->dim, ns = mp->nspecies;
    int rc;
    // rho and rhotot are the reference's correction_flux arguments; the
    // correction itself reads only the fluxes, so they are checked when given
    if (rho && (rc = check_mf(ctx, rho, 0))) return rc;
    if (rhotot && (rc = check_mf(ctx, rhotot, 0))) return rc;
    if ((rc = check_mf(ctx, stoch_mass_fluxdiv, 0)) || (rc = check_ncomp(*stoch_mass_fluxdiv, ns))) return rc;
    for (int d = 0; d < dim; d++) {
        if ((rc = check_mf(ctx, &sqrtLonsager_fc[d], 0)) || (rc = check_ncomp(sqrtLonsager_fc[d], ns * ns))) return rc;
        if (stoch_mass_flux && ((rc = check_mf(ctx, &stoch_mass_flux[d], 0)) ||
                                (rc = check_ncomp(stoch_mass_flux[d], ns))))
            return rc;
    }
    for (int q = 0; q < n_rngs * dim; q++)
        if ((rc = check_mf(ctx, &W_fc[q], 0)) || (rc = check_ncomp(W_fc[q], ns))) return rc;
    const int nL = dim * ns * ns, nW = n_rngs * dim * ns, nF = dim * ns;
    DevArrays A;
    if ((rc = A.alloc(nL + nW + ns + nF, ctx->g0.nc))) return rc;
    double** d_L = A.a.data();
    double** d_W = d_L + nL;
    double** d_div = d_W + nW;
    double** d_F = d_div + ns;
    for (int d = 0; d < dim; d++)
        if ((rc = mf_comps_to_dev(ctx, sqrtLonsager_fc[d], ns * ns, d_L + d * ns * ns))) return rc;
    // W_fc[r*dim + d] holds the ns species components of stage r, direction d
    for (int q = 0; q < n_rngs * dim; q++)
        if ((rc = mf_comps_to_dev(ctx, W_fc[q], ns, d_W + q * ns))) return rc;
    if (increment && (rc = mf_comps_to_dev(ctx, *stoch_mass_fluxdiv, ns, d_div))) return rc;
    std::vector<const double*> cL(d_L, d_L + nL), cW(d_W, d_W + nW);
    if ((rc = fhd_dev_stochastic_mass_fluxdiv(ctx, mp, sp, cL.data(), dt, weights, n_rngs, cW.data(), increment,
                                              d_div, d_F)))
        return rc;
    std::vector<const double*> cdiv(d_div, d_div + ns);
    if ((rc = dev_to_mf_comps(ctx, cdiv.data(), ns, *stoch_mass_fluxdiv))) return rc;
    if (stoch_mass_flux)
        for (int d = 0; d < dim; d++) {
            std::vector<const double*> src(d_F + d * ns, d_F + (d + 1) * ns);
            if ((rc = dev_to_mf_comps(ctx, src.data(), ns, stoch_mass_flux[d]))) return rc;
        }
    return 0;
}

}  // extern "C"
