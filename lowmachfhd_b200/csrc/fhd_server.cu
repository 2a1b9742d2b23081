// fhd_server.cu -- device-resident serving of Stokes / timestep requests,
// and the counter-based device random number generator the served
// requests draw their stochastic fields from.
//
// The reference has no serving layer: one driver runs one problem
// (src_lowMach/main_driver.f90).  Here a request is one problem -- a grid,
// a fluid or mixture, a number of overdamped or inertial timesteps
// (advance_timestep_overdamped.f90 / advance_timestep_inertial.f90) -- and
// the server runs many of them at once on one GPU:
//
//  * worker threads, each with its own non-blocking CUDA stream and one
//    request at a time (a request's GMRES synchronises only its stream);
//  * admission in arrival order while the request's device bytes fit in
//    the HBM budget next to the requests already running (continuous
//    batching: a finished request frees its slot and bytes at once);
//  * request state (velocity, densities, pressure, coefficients, noise)
//    allocated stream-ordered and resident for all of its steps;
//  * stochastic fields from Philox-4x32-10 keyed by the request's seed and
//    counted by (step, field, element), so a result depends only on the
//    request and never on what runs beside it.
//
// The admission policy (Sched) is plain C++ without CUDA so that it can be
// exercised on a host without a GPU (fhd_sched_simulate).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "fhd_solver.cuh"

namespace fhd {

// requests of at least this many steps run with GMRES iteration graphs
constexpr int SERVE_ITER_GRAPH_STEPS = 16;

int advance_overdamped(fhd_ctx* ctx, const fhd_stoch_params* sp, const fhd_mixture_params* mp, double dt,
                       double* const umac[], double* const rho[], double* pi, const double* eta,
                       const double* const eta_ed[], const double* kappa, const double* temperature,
                       const double* const temperature_ed[], const double* const W_cc[], const double* const W_ed[],
                       const double* const W_mass[], fhd_solve_stats* stats2);
int advance_inertial_ms(fhd_ctx* ctx, const fhd_stoch_params* sp, const fhd_mixture_params* mp, double dt,
                        double* const umac[], double* const rho[], double* pi, double* const fluxdiv[],
                        const double* eta, const double* const eta_ed[], const double* kappa,
                        const double* temperature, const double* const temperature_ed[], const double* const W_cc[],
                        const double* const W_ed[], const double* const W_mass[], fhd_solve_stats* stats2);

// ---------------------------------------------------------------------
// Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC 2011): ten rounds of two 32x32->64 multiplies with
// the key bumped by the Weyl constants between rounds
// ---------------------------------------------------------------------
struct U4 {
    uint32_t x, y, z, w;
};

__host__ __device__ __forceinline__ void mulhilo32(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
    const uint64_t p = (uint64_t)a * (uint64_t)b;
    hi = (uint32_t)(p >> 32);
    lo = (uint32_t)p;
}

__host__ __device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo32(0xD2511F53u, c.x, hi0, lo0);
        mulhilo32(0xCD9E8D57u, c.z, hi1, lo1);
        c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

// N(0,1) pairs by the Box-Muller transform of two 53-bit uniforms taken from
// one Philox block; element 2j and 2j+1 of a field share the counter
// (j, field, stream_a, stream_b)
__global__ void __launch_bounds__(256) k_normal(double* out, i64 n, uint64_t seed, uint32_t field, uint32_t sa,
                                                uint32_t sb, double scale) {
    const i64 pairs = (n + 1) / 2;
    for (i64 j = blockIdx.x * (i64)blockDim.x + threadIdx.x; j < pairs; j += (i64)gridDim.x * blockDim.x) {
        const U4 r = philox4x32_10(U4{(uint32_t)j, field, sa, sb}, (uint32_t)seed, (uint32_t)(seed >> 32));
        const uint64_t a = ((uint64_t)r.x << 32) | r.y, b = ((uint64_t)r.z << 32) | r.w;
        const double u1 = (double)((a >> 11) + 1) * 0x1.0p-53;  // (0, 1]
        const double u2 = (double)(b >> 11) * 0x1.0p-53;        // [0, 1)
        const double rad = sqrt(-2.0 * log(u1));
        double s, c;
        sincospi(2.0 * u2, &s, &c);
        out[2 * j] = scale * rad * c;
        if (2 * j + 1 < n) out[2 * j + 1] = scale * rad * s;
    }
}

__global__ void __launch_bounds__(256) k_fill(double* out, i64 n, double v) {
    for (i64 f = blockIdx.x * (i64)blockDim.x + threadIdx.x; f < n; f += (i64)gridDim.x * blockDim.x) out[f] = v;
}

// sum of squares of the velocity components (a request's result digest)
__global__ void __launch_bounds__(RED_THREADS) k_sumsq(i64 n, int ncomp, CSVec<double> u, RedSlot rs) {
    double s = 0.0;
    for (i64 f = blockIdx.x * (i64)blockDim.x + threadIdx.x; f < n; f += (i64)gridDim.x * blockDim.x)
        for (int c = 0; c < ncomp; c++) s += u.c[c][f] * u.c[c][f];
    red_finish(s, rs);
}

// ---------------------------------------------------------------------
// admission policy
// ---------------------------------------------------------------------
struct Sched {
    int slots = 1;
    uint64_t budget = 0;
    uint64_t used = 0;
    int running = 0;
    // the head of the queue may start now
    bool admits(uint64_t bytes) const { return running < slots && used + bytes <= budget; }
    void start(uint64_t bytes) {
        used += bytes;
        running++;
    }
    void finish(uint64_t bytes) {
        used -= bytes;
        running--;
    }
};

// device bytes a request holds: its context (multigrid hierarchy, Krylov
// storage, step work arrays, mass-flux work arrays) and its own state and
// noise.  An upper estimate from the allocation sizes.
static uint64_t request_bytes(const fhd_request* r) {
    const int dim = r->dim, nE = dim == 2 ? 1 : 3, ns = r->nspecies;
    uint64_t nc = 1;
    for (int d = 0; d < dim; d++) nc *= (uint64_t)r->n_cells[d];
    const int m = r->params.gmres_max_inner;
    const double s = r->precision == FHD_PREC_MIXED ? 4.0 : 8.0;
    // multigrid: per level phi, rhs, tmp, alpha (dim each), beta, gamma,
    // edges, in mixed 3D the row-tile smoother's diagonal (dim); cc: a (dim),
    // phi, rhs, tmp; level sums to 8/7 (3D) or 4/3 (2D)
    const double lv = dim == 3 ? 8.0 / 7.0 : 4.0 / 3.0;
    const double rbx = (r->precision == FHD_PREC_MIXED && dim == 3) ? dim : 0;
    const double mg = (4.0 * dim + 2 + nE + dim + 3 + 2 * dim + 1 + rbx) * s * lv;
    const double krylov = (double)(m + 1 + 4) * (dim + 1) * 8.0;
    const double step = (39.0 + ns * (2 + dim)) * 8.0;
    const double mass = ns > 1 ? (ns * ns + ns + dim * ns) * s : 0.0;
    const double state = (dim + ns + 1 + 1 + nE + 1 + 1 + nE + ns) * 8.0;
    const double noise = (2.0 * dim + 2.0 * nE + 2.0 * dim * ns) * 8.0;
    return (uint64_t)((mg + krylov + step + mass + state + noise) * (double)nc) + (64ull << 20);
}

// ---------------------------------------------------------------------
// the server
// ---------------------------------------------------------------------
struct Pending {
    long long id;
    fhd_request req;
    uint64_t bytes;
    double t_submit;
};

struct Server {
    int device = 0;
    Sched sched;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Pending> queue;
    std::map<long long, fhd_request_result> done;
    std::vector<std::thread> workers;
    bool stop = false;
    long long next_id = 1;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

static int run_request(const fhd_request& q, cudaStream_t st, fhd_request_result& res) {
    const int dim = q.dim;
    if (dim < 2 || dim > 3) return FHD_ERR_BAD_ARG;
    const int nE = dim == 2 ? 1 : 3;
    const int ns = q.nspecies;
    if (ns < 1 || ns > 5 || q.steps < 0 || !(q.dt > 0.0) || (ns > 1 && q.mix.nspecies != ns))
        return FHD_ERR_BAD_ARG;
    fhd_ctx* ctx = nullptr;
    const double dx3[3] = {q.dx, q.dx, q.dx};
    int rc = fhd_ctx_create(dim, q.n_cells, dx3, q.visc_type, &q.params, q.precision, &ctx);
    if (rc) return rc;
    fhd_ctx_set_stream(ctx, st);
    // whole GMRES iterations as graphs once a request is long enough to
    // amortise their capture (a short request would pay more in capture and
    // instantiation than its replays save)
    if (q.steps >= SERVE_ITER_GRAPH_STEPS) fhd_ctx_set_graphs(ctx, 2);
    i64 nc = 1;
    for (int d = 0; d < dim; d++) nc *= q.n_cells[d];
    // state and noise, stream-ordered on the worker's stream
    std::vector<double*> blocks;
    auto alloc = [&]() -> double* {
        void* p = nullptr;
        if (cudaMallocAsync(&p, sizeof(double) * nc, st) != cudaSuccess) return nullptr;
        blocks.push_back((double*)p);
        return (double*)p;
    };
    double *umac[3] = {nullptr, nullptr, nullptr};
    double *rho[FHD_MAX_SPECIES] = {nullptr}, *fdiv[FHD_MAX_SPECIES] = {nullptr};
    double *eta_ed[3] = {nullptr, nullptr, nullptr}, *T_ed[3] = {nullptr, nullptr, nullptr};
    double *Wcc[6] = {nullptr}, *Wed[12] = {nullptr}, *Wm[30] = {nullptr};
    double *pi = nullptr, *eta = nullptr, *kappa = nullptr, *T = nullptr;
    bool ok = true;
    for (int c = 0; c < dim; c++) ok = ok && (umac[c] = alloc());
    for (int s = 0; s < ns; s++) ok = ok && (rho[s] = alloc()) && (fdiv[s] = alloc());
    ok = ok && (pi = alloc()) && (eta = alloc()) && (kappa = alloc()) && (T = alloc());
    for (int e = 0; e < nE; e++) ok = ok && (eta_ed[e] = alloc()) && (T_ed[e] = alloc());
    const int nstage = 2;
    for (int i = 0; i < nstage * dim; i++) ok = ok && (Wcc[i] = alloc());
    for (int i = 0; i < nstage * nE; i++) ok = ok && (Wed[2 * i] = alloc());
    if (ns > 1)
        for (int i = 0; i < nstage * dim * ns; i++) ok = ok && (Wm[i] = alloc());
    // the symmetric stress form uses equal edge components
    for (int i = 0; i < nstage * nE; i++) Wed[2 * i + 1] = Wed[2 * i];
    const int nb = flat_blocks(nc);
    auto fill = [&](double* p, double v) { k_fill<<<nb, 256, 0, st>>>(p, nc, v); };
    if (ok) {
        for (int c = 0; c < dim; c++) fill(umac[c], 0.0);
        for (int s = 0; s < ns; s++) {
            fill(rho[s], q.rho0 / ns);
            fill(fdiv[s], 0.0);
        }
        fill(pi, 0.0);
        fill(eta, q.eta);
        fill(kappa, 0.0);
        fill(T, 1.0);
        for (int e = 0; e < nE; e++) {
            fill(eta_ed[e], q.eta);
            fill(T_ed[e], 1.0);
        }
        if (cudaPeekAtLastError() != cudaSuccess) ok = false;
    }
    if (!ok) rc = FHD_ERR_OOM;
    fhd_stoch_params sp;
    memset(&sp, 0, sizeof(sp));
    sp.k_B = q.kT;
    sp.variance_coef_mom = 1.0;
    sp.dV = dim == 3 ? q.dx * q.dx * q.dx : q.dx * q.dx * q.cell_depth;
    sp.stoch_stress_form = 1;
    const fhd_mixture_params* mp = ns > 1 ? &q.mix : nullptr;
    // Stochastic fields.  Momentum: field ids 0.. (cell stages, then edge
    // stages) counted by the step.  Mass: field ids 1000 + (d*ns + i)
    // counted by the noise index j: the overdamped step draws M_2k and
    // M_2k+1 for its two stages; the inertial step k uses M_{k-1} in the
    // predictor and M_k in the corrector (the predictor reuses the previous
    // corrector's fields, advance_timestep_inertial.f90), with F^0 from M_0.
    auto normal = [&](double* p, uint32_t field, uint32_t count, double scale) {
        k_normal<<<nb, 256, 0, st>>>(p, nc, q.seed, field, count, 0x5eedu, scale);
    };
    auto mass_stage = [&](int stage, uint32_t j) {
        for (int i = 0; i < dim * ns; i++) normal(Wm[stage * dim * ns + i], 1000u + i, j, 1.0);
    };
    auto draw = [&](int step) {
        uint32_t slot = 0;
        for (int i = 0; i < nstage * dim; i++) normal(Wcc[i], slot++, (uint32_t)step, std::sqrt(2.0));
        for (int i = 0; i < nstage * nE; i++) normal(Wed[2 * i], slot++, (uint32_t)step, 1.0);
        if (ns > 1) {
            if (q.kind == FHD_REQ_INERTIAL) {
                mass_stage(0, (uint32_t)(step - 1));
                mass_stage(1, (uint32_t)step);
            } else {
                mass_stage(0, (uint32_t)(2 * step));
                mass_stage(1, (uint32_t)(2 * step + 1));
            }
        }
    };
    int iters = 0, worst = 0;
    if (!rc && q.kind == FHD_REQ_INERTIAL && ns > 1) {
        // F^0 at start-up (main_driver.f90 before the time loop)
        mass_stage(0, 0u);
        const double w1[1] = {1.0};
        const double* cr[FHD_MAX_SPECIES];
        for (int s = 0; s < ns; s++) cr[s] = rho[s];
        rc = mass_fluxdiv(ctx, mp, &sp, cr, q.dt, w1, 1, Wm, fdiv);
    }
    for (int step = 1; step <= q.steps && rc >= 0; step++) {
        draw(step);
        fhd_solve_stats s2[2];
        memset(s2, 0, sizeof(s2));
        int r2;
        if (q.kind == FHD_REQ_INERTIAL) {
            r2 = advance_inertial_ms(ctx, &sp, mp, q.dt, umac, rho, pi, fdiv, eta, eta_ed, kappa, T, T_ed, Wcc, Wed,
                                     ns > 1 ? Wm : nullptr, s2);
        } else {
            r2 = advance_overdamped(ctx, &sp, mp, q.dt, umac, rho, pi, eta, eta_ed, kappa, T, T_ed, Wcc, Wed,
                                    ns > 1 ? Wm : nullptr, s2);
        }
        if (r2 < 0) {
            rc = r2;
            break;
        }
        worst = std::max(worst, r2);
        iters += s2[0].total_iters + s2[1].total_iters;
    }
    if (rc >= 0) {
        CSVec<double> u;
        for (int c = 0; c < 4; c++) u.c[c] = c < dim ? umac[c] : nullptr;
        k_sumsq<<<nb, RED_THREADS, 0, st>>>(nc, dim, u, slot(ctx, S_NRM));
        if (sync_scalars(ctx, S_NRM, 1)) rc = FHD_ERR_CUDA;
        res.u_sumsq = ctx->hscal[S_NRM];
        if (q.out_umac)
            for (int c = 0; c < dim && rc >= 0; c++)
                if (cudaMemcpyAsync(q.out_umac + (i64)c * nc, umac[c], sizeof(double) * nc, cudaMemcpyDeviceToHost,
                                    st) != cudaSuccess)
                    rc = FHD_ERR_CUDA;
        if (q.out_rho)
            for (int s = 0; s < ns && rc >= 0; s++)
                if (cudaMemcpyAsync(q.out_rho + (i64)s * nc, rho[s], sizeof(double) * nc, cudaMemcpyDeviceToHost,
                                    st) != cudaSuccess)
                    rc = FHD_ERR_CUDA;
        if (cudaStreamSynchronize(st) != cudaSuccess) rc = FHD_ERR_CUDA;
    }
    res.gmres_iters = iters;
    res.launches = fhd_ctx_kernel_launches(ctx);
    for (double* p : blocks) cudaFreeAsync(p, st);
    cudaStreamSynchronize(st);
    fhd_ctx_destroy(ctx);
    return rc < 0 ? rc : worst;
}

static void worker_main(Server* S) {
    cudaSetDevice(S->device);
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) st = nullptr;
    for (;;) {
        Pending p;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            // queued requests are finished before a stop takes effect
            S->cv_work.wait(lk, [&] {
                return (!S->queue.empty() && S->sched.admits(S->queue.front().bytes)) ||
                       (S->stop && S->queue.empty());
            });
            if (S->queue.empty()) break;
            p = S->queue.front();
            S->queue.pop_front();
            S->sched.start(p.bytes);
        }
        fhd_request_result res;
        memset(&res, 0, sizeof(res));
        res.id = p.id;
        res.t_submit = p.t_submit;
        res.t_start = S->now();
        res.bytes = p.bytes;
        res.status = st ? run_request(p.req, st, res) : FHD_ERR_CUDA;
        res.t_end = S->now();
        {
            std::lock_guard<std::mutex> lk(S->mu);
            S->sched.finish(p.bytes);
            S->done[p.id] = res;
        }
        S->cv_work.notify_all();
        S->cv_done.notify_all();
    }
    if (st) cudaStreamDestroy(st);
}

}  // namespace fhd

using namespace fhd;

struct fhd_server {
    Server s;
};

extern "C" {

int fhd_dev_fill_normal(double* out, long long n, unsigned long long seed, unsigned field, unsigned stream_a,
                        unsigned stream_b, double scale, void* stream) {
    if (!out || n < 0) return FHD_ERR_BAD_ARG;
    if (n == 0) return FHD_OK;
    k_normal<<<flat_blocks((n + 1) / 2), 256, 0, (cudaStream_t)stream>>>(out, n, seed, field, stream_a, stream_b,
                                                                         scale);
    FHD_CUDA_TRY(cudaPeekAtLastError());
    return FHD_OK;
}

void fhd_philox4x32_10(const unsigned ctr[4], const unsigned key[2], unsigned out[4]) {
    const U4 r = philox4x32_10(U4{ctr[0], ctr[1], ctr[2], ctr[3]}, key[0], key[1]);
    out[0] = r.x;
    out[1] = r.y;
    out[2] = r.z;
    out[3] = r.w;
}

unsigned long long fhd_request_bytes(const fhd_request* r) { return r ? request_bytes(r) : 0ull; }

void fhd_request_default(fhd_request* r) {
    memset(r, 0, sizeof(*r));
    r->kind = FHD_REQ_OVERDAMPED;
    r->dim = 2;
    r->n_cells[0] = r->n_cells[1] = 64;
    r->n_cells[2] = 1;
    r->dx = 1.0;
    r->cell_depth = 1.0;
    r->visc_type = 1;
    r->precision = FHD_PREC_MIXED;
    r->nspecies = 1;
    r->rho0 = 1.0;
    r->eta = 1.0;
    r->kT = 1.0;
    r->dt = 0.1;
    r->steps = 1;
    r->seed = 1;
    fhd_gmres_params_default(&r->params);
}

int fhd_server_create(int slots, unsigned long long hbm_budget_bytes, fhd_server** out) {
    if (!out || slots < 1 || slots > 64) return FHD_ERR_BAD_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return FHD_ERR_NO_DEVICE;
    fhd_server* sv = new fhd_server();
    cudaGetDevice(&sv->s.device);
    // Requests allocate their state stream-ordered from the device's default
    // pool.  Its default release threshold (0) hands every freed block back
    // at the next synchronisation, so each request would map its memory
    // again; keeping up to the budget in the pool makes admission cheap.
    // A process-local allocator attribute, not a device setting.
    {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, sv->s.device) == cudaSuccess) {
            unsigned long long thr = hbm_budget_bytes;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
    }
    sv->s.sched.slots = slots;
    sv->s.sched.budget = hbm_budget_bytes;
    for (int i = 0; i < slots; i++) sv->s.workers.emplace_back(worker_main, &sv->s);
    *out = sv;
    return FHD_OK;
}

int fhd_server_submit(fhd_server* sv, const fhd_request* req, long long* id) {
    if (!sv || !req || !id) return FHD_ERR_BAD_ARG;
    const uint64_t b = request_bytes(req);
    if (b > sv->s.sched.budget) {
        set_last_error("fhd_server_submit: the request needs more device memory than the whole budget");
        return FHD_ERR_OOM;
    }
    {
        std::lock_guard<std::mutex> lk(sv->s.mu);
        Pending p;
        p.id = sv->s.next_id++;
        p.req = *req;
        p.bytes = b;
        p.t_submit = sv->s.now();
        sv->s.queue.push_back(p);
        *id = p.id;
    }
    sv->s.cv_work.notify_all();
    return FHD_OK;
}

int fhd_server_wait(fhd_server* sv, long long id, fhd_request_result* res) {
    if (!sv || !res) return FHD_ERR_BAD_ARG;
    std::unique_lock<std::mutex> lk(sv->s.mu);
    sv->s.cv_done.wait(lk, [&] { return sv->s.done.count(id) > 0; });
    *res = sv->s.done[id];
    sv->s.done.erase(id);
    return FHD_OK;
}

double fhd_server_clock(fhd_server* sv) { return sv ? sv->s.now() : 0.0; }

int fhd_server_destroy(fhd_server* sv) {
    if (!sv) return FHD_OK;
    {
        std::lock_guard<std::mutex> lk(sv->s.mu);
        sv->s.stop = true;
    }
    sv->s.cv_work.notify_all();
    for (auto& t : sv->s.workers) t.join();
    delete sv;
    return FHD_OK;
}

// The admission policy on a synthetic trace, without a GPU: n requests
// with arrival times, device bytes and run times; returns each start time
// (event simulation of the worker pool above).
int fhd_sched_simulate(int slots, unsigned long long budget, int n, const double* arrive,
                       const unsigned long long* bytes, const double* runtime, double* start) {
    if (slots < 1 || n < 0 || (n > 0 && (!arrive || !bytes || !runtime || !start))) return FHD_ERR_BAD_ARG;
    for (int i = 0; i < n; i++)
        if (bytes[i] > budget) return FHD_ERR_OOM;
    Sched S;
    S.slots = slots;
    S.budget = budget;
    std::vector<std::pair<double, int>> running;  // (end time, request)
    int head = 0;
    double t = 0.0;
    while (head < n) {
        const bool idle = running.empty();
        const double next_end = idle ? 0.0 : std::min_element(running.begin(), running.end())->first;
        if (arrive[head] > t && (idle || arrive[head] <= next_end)) t = std::max(t, arrive[head]);
        if (arrive[head] <= t && S.admits(bytes[head])) {
            start[head] = t;
            S.start(bytes[head]);
            running.push_back({t + runtime[head], head});
            head++;
            continue;
        }
        // advance to the next completion
        if (idle) return FHD_ERR_BAD_ARG;
        auto it = std::min_element(running.begin(), running.end());
        t = std::max(t, it->first);
        S.finish(bytes[it->second]);
        running.erase(it);
    }
    return FHD_OK;
}

}  // extern "C"
