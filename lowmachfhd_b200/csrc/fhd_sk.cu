// fhd_sk.cu -- static structure factors on the device: the analysis that
// HydroGrid's updateStructureFactors (HydroGrid/HydroGridModule.f90:
// 1077-1180) runs on the host every sampled step, here as one cuFFT
// real-to-complex transform per variable and one kernel that applies the
// staggered-velocity phase shift (HydroGridModule.f90:1119-1141) and folds
// every pair's spectrum into its running mean (1160-1180).  The fields stay
// in HBM: nothing crosses PCIe until the caller reads the spectra.
//
// Layout: a variable is a cell or face array in the canonical order (x
// fastest); its transform is the half spectrum kx = 0 .. nx/2 of the
// unnormalised forward DFT, index (kz, ky, kx), kx fastest.  Integer
// wavenumbers follow the FFT order 0, 1, .., -2, -1.
#include <cuda_runtime.h>
#include <cufft.h>

#include <cstring>
#include <string>
#include <vector>

#include "fhd_solver.cuh"

namespace fhd {

constexpr int SK_MAXVARS = 8;
constexpr int SK_MAXPAIRS = 16;

struct SkPairs {
    int a[SK_MAXPAIRS], b[SK_MAXPAIRS];
    int shift[SK_MAXVARS];  // phase sign (-1, 0, +1) of each variable
    int dir[SK_MAXVARS];    // its direction (face-centred velocity component)
};

// one sample: per half-spectrum mode, the phase-shifted transforms of the
// variables, then S_p = ((n-1) S_p + Ua conj(Ub)) / n for every pair
__global__ void __launch_bounds__(256) k_sk_update(i64 nm, int nxh, int ny, int nx, int nz, int nvars, int npairs,
                                                   SkPairs P, const cufftDoubleComplex* __restrict__ U,
                                                   double* __restrict__ S, double nsamp) {
    for (i64 m = blockIdx.x * (i64)blockDim.x + threadIdx.x; m < nm; m += (i64)gridDim.x * blockDim.x) {
        const int ix = (int)(m % nxh);
        const i64 r = m / nxh;
        const int iy = (int)(r % ny), iz = (int)(r / ny);
        const int kw[3] = {ix <= nx / 2 ? ix : ix - nx, iy <= ny / 2 ? iy : iy - ny, iz <= nz / 2 ? iz : iz - nz};
        const int nn[3] = {nx, ny, nz};
        double re[SK_MAXVARS], im[SK_MAXVARS];
        for (int v = 0; v < nvars; v++) {
            const cufftDoubleComplex u = U[(i64)v * nm + m];
            re[v] = u.x;
            im[v] = u.y;
            if (P.shift[v] != 0) {
                // exp(i s k_d pi / N_d)
                double sn, cs;
                sincospi((double)(P.shift[v] * kw[P.dir[v]]) / (double)nn[P.dir[v]], &sn, &cs);
                const double x = re[v] * cs - im[v] * sn, y = re[v] * sn + im[v] * cs;
                re[v] = x;
                im[v] = y;
            }
        }
        for (int p = 0; p < npairs; p++) {
            const int a = P.a[p], b = P.b[p];
            // Ua conj(Ub)
            const double cr = re[a] * re[b] + im[a] * im[b];
            const double ci = im[a] * re[b] - re[a] * im[b];
            double* sp = S + (i64)2 * p * nm;
            sp[m] = ((nsamp - 1.0) * sp[m] + cr) / nsamp;
            sp[nm + m] = ((nsamp - 1.0) * sp[nm + m] + ci) / nsamp;
        }
    }
}

}  // namespace fhd

using namespace fhd;

struct fhd_sk {
    int dim = 3;
    int n[3] = {1, 1, 1};
    double dV = 1.0;
    int nvars = 0, npairs = 0;
    SkPairs P;
    i64 nc = 0, nm = 0;  // cells, half-spectrum modes
    cufftHandle plan = 0;
    bool planned = false;
    double* real = nullptr;               // staged copy of one variable
    cufftDoubleComplex* U = nullptr;      // nvars transforms
    double* S = nullptr;                  // npairs running means (re block, im block)
    long long samples = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev = nullptr;  // orders the object's stream with the caller's
};

extern "C" {

int fhd_sk_create(int dim, const int n_cells[3], double dV, int nvars, const int* shift, int npairs,
                  const int* pairs, fhd_sk** out) {
    if (!out || !n_cells || !pairs || (dim != 2 && dim != 3) || nvars < 1 || nvars > SK_MAXVARS || npairs < 1 ||
        npairs > SK_MAXPAIRS || !(dV > 0.0))
        return FHD_ERR_BAD_ARG;
    *out = nullptr;
    for (int d = 0; d < dim; d++)
        if (n_cells[d] < 2) return FHD_ERR_BAD_ARG;
    for (int p = 0; p < 2 * npairs; p++)
        if (pairs[p] < 0 || pairs[p] >= nvars) return FHD_ERR_BAD_ARG;
    if (shift)
        for (int v = 0; v < nvars; v++)
            if (shift[v] < -1 || shift[v] > 1 || (shift[v] != 0 && v >= dim)) return FHD_ERR_BAD_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return FHD_ERR_NO_DEVICE;
    fhd_sk* s = new fhd_sk();
    s->dim = dim;
    for (int d = 0; d < 3; d++) s->n[d] = d < dim ? n_cells[d] : 1;
    s->dV = dV;
    s->nvars = nvars;
    s->npairs = npairs;
    memset(&s->P, 0, sizeof s->P);
    for (int p = 0; p < npairs; p++) {
        s->P.a[p] = pairs[2 * p];
        s->P.b[p] = pairs[2 * p + 1];
    }
    for (int v = 0; v < nvars; v++) {
        s->P.shift[v] = shift ? shift[v] : 0;
        s->P.dir[v] = v < dim ? v : 0;
    }
    s->nc = (i64)s->n[0] * s->n[1] * s->n[2];
    s->nm = (i64)(s->n[0] / 2 + 1) * s->n[1] * s->n[2];
    int rc = FHD_OK;
    auto fail = [&](int code, const char* what) {
        set_last_error(std::string("fhd_sk_create: ") + what);
        rc = code;
    };
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->ev, cudaEventDisableTiming) != cudaSuccess)
        fail(FHD_ERR_CUDA, "stream");
    if (!rc && (cudaMalloc(&s->real, sizeof(double) * s->nc) != cudaSuccess ||
                cudaMalloc(&s->U, sizeof(cufftDoubleComplex) * s->nm * nvars) != cudaSuccess ||
                cudaMalloc(&s->S, sizeof(double) * 2 * s->nm * npairs) != cudaSuccess))
        fail(FHD_ERR_OOM, "device memory");
    if (!rc && cudaMemsetAsync(s->S, 0, sizeof(double) * 2 * s->nm * npairs, s->stream) != cudaSuccess)
        fail(FHD_ERR_CUDA, "memset");
    if (!rc) {
        // cuFFT dimensions slowest first: (nz,) ny, nx
        const cufftResult r = dim == 3 ? cufftPlan3d(&s->plan, s->n[2], s->n[1], s->n[0], CUFFT_D2Z)
                                       : cufftPlan2d(&s->plan, s->n[1], s->n[0], CUFFT_D2Z);
        if (r != CUFFT_SUCCESS) fail(FHD_ERR_CUDA, "cufftPlan");
        else s->planned = true;
    }
    if (!rc && cufftSetStream(s->plan, s->stream) != CUFFT_SUCCESS) fail(FHD_ERR_CUDA, "cufftSetStream");
    if (!rc && cudaStreamSynchronize(s->stream) != cudaSuccess) fail(FHD_ERR_CUDA, "synchronize");
    if (rc) {
        fhd_sk_destroy(s);
        return rc;
    }
    *out = s;
    return FHD_OK;
}

int fhd_sk_update(fhd_sk* s, const double* const vars[], void* stream) {
    if (!s || !vars) return FHD_ERR_BAD_ARG;
    for (int v = 0; v < s->nvars; v++)
        if (!vars[v]) return FHD_ERR_BAD_ARG;
    // order after the caller's work on its stream
    if (stream) {
        FHD_CUDA_TRY(cudaEventRecord(s->ev, (cudaStream_t)stream));
        FHD_CUDA_TRY(cudaStreamWaitEvent(s->stream, s->ev, 0));
    }
    for (int v = 0; v < s->nvars; v++) {
        // the transform reads a staged copy, so the caller's field is never
        // touched whatever cuFFT does with its input
        FHD_CUDA_TRY(cudaMemcpyAsync(s->real, vars[v], sizeof(double) * s->nc, cudaMemcpyDeviceToDevice, s->stream));
        if (cufftExecD2Z(s->plan, s->real, s->U + (i64)v * s->nm) != CUFFT_SUCCESS) {
            set_last_error("fhd_sk_update: cufftExecD2Z failed");
            return FHD_ERR_CUDA;
        }
    }
    s->samples++;
    const int nxh = s->n[0] / 2 + 1;
    k_sk_update<<<flat_blocks(s->nm), 256, 0, s->stream>>>(s->nm, nxh, s->n[1], s->n[0], s->n[2], s->nvars,
                                                           s->npairs, s->P, s->U, s->S, (double)s->samples);
    FHD_CUDA_TRY(cudaPeekAtLastError());
    // the caller's stream waits for this sample before it overwrites the fields
    if (stream) {
        FHD_CUDA_TRY(cudaEventRecord(s->ev, s->stream));
        FHD_CUDA_TRY(cudaStreamWaitEvent((cudaStream_t)stream, s->ev, 0));
    }
    return FHD_OK;
}

int fhd_sk_read(fhd_sk* s, int pair, double* re, double* im, long long* samples) {
    if (!s || pair < 0 || pair >= s->npairs) return FHD_ERR_BAD_ARG;
    FHD_CUDA_TRY(cudaStreamSynchronize(s->stream));
    // HydroGridModule.f90:1862-1868: 1/n_fft_cells * dV (structFactMultiplier 1)
    const double scale = s->dV / (double)s->nc;
    std::vector<double> h((size_t)s->nm);
    double* dst[2] = {re, im};
    for (int part = 0; part < 2; part++) {
        if (!dst[part]) continue;
        FHD_CUDA_TRY(cudaMemcpy(h.data(), s->S + ((i64)2 * pair + part) * s->nm, sizeof(double) * s->nm,
                                cudaMemcpyDeviceToHost));
        for (i64 m = 0; m < s->nm; m++) dst[part][m] = h[(size_t)m] * scale;
    }
    if (samples) *samples = s->samples;
    return FHD_OK;
}

long long fhd_sk_modes(fhd_sk* s) { return s ? (long long)s->nm : 0; }

int fhd_sk_destroy(fhd_sk* s) {
    if (!s) return FHD_OK;
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->planned) cufftDestroy(s->plan);
    cudaFree(s->real);
    cudaFree(s->U);
    cudaFree(s->S);
    if (s->ev) cudaEventDestroy(s->ev);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return FHD_OK;
}

}  // extern "C"
