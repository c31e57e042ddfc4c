// vs_spectrum.cu -- formants of listener traces on the device.
//
// Restates get_formants_bw (results/formants_bandwidths.py:5-80) for a batch
// of traces: level = 10 log10 |FFT(x)|^2 over the full spectrum (double,
// cuFFT real-to-complex, the upper half mirrored), frequency axis
// f_k = k fs / (N - 1); scan the bins from 1 for local maxima; at each peak
// walk left and right while the level stays above peak - 3 dB, take the
// crossing frequencies as numpy.interp of the two bins around each crossing
// (numpy's two-point rules, including its result for the decreasing pair on
// the right side), record (bandwidth, centre frequency, peak level) and
// resume at the right crossing.  One thread scans one trace; the scan is
// sequential by definition (each peak's window moves the cursor).
#include <cuda_runtime.h>
#include <cufft.h>

#include <cmath>
#include <string>

#include "vs_device.h"

namespace vsb {
namespace {

__global__ void to_double_kernel(const float* __restrict__ x, double* __restrict__ y, int64_t count) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < count) y[i] = (double)x[i];
}

// level of bins 0 .. N/2 of every trace (N/2 + 1 complex values per trace)
__global__ void level_kernel(const cufftDoubleComplex* __restrict__ X, double* __restrict__ level, int64_t n,
                             int64_t nh, int ntr) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nh * ntr) return;
    const int64_t t = i / nh, k = i % nh;
    const double a = hypot(X[i].x, X[i].y);
    level[t * n + k] = 10.0 * log10(a * a);
}

// numpy.interp(x, [x0, x1], [f0, f1]) for a two-point table, as numpy
// evaluates it (binary_search_with_guess + the interpolation branch).
__device__ double interp2(double x, double x0, double x1, double f0, double f1) {
    if (isnan(x)) return x;
    if (x > x1) return f1;
    if (x < x0) return f0;
    // linear search of a short table: j = 0 unless x >= x1
    if (x >= x1) return f1;
    if (x0 == x) return f0;
    const double slope = (f1 - f0) / (x1 - x0);
    double r = slope * (x - x0) + f0;
    if (isnan(r)) {
        r = slope * (x - x1) + f1;
        if (isnan(r) && f0 == f1) r = f0;
    }
    return r;
}

__global__ void formant_scan_kernel(const double* __restrict__ level, int64_t n, double fs, int nf,
                                    double* __restrict__ out, int ntr) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntr) return;
    const double* L = level + (int64_t)t * n;
    // the upper half of the spectrum of a real signal mirrors the lower half
    auto lev = [&](int64_t k) { return k <= n / 2 ? L[k] : L[n - k]; };
    const double df = fs / (double)(n - 1);
    auto freq = [&](int64_t k) { return (double)k * df; };
    double* o = out + (int64_t)t * 3 * nf;
    for (int j = 0; j < 3 * nf; ++j) o[j] = 0.0;
    int found = 0;
    int64_t i = 1;
    while (found < nf && i < n - 1) {
        const double li = lev(i);
        if (li > lev(i - 1) && li > lev(i + 1)) {
            const double cut = li - 3.0;
            int64_t lo = i;
            while (lo > 0 && lev(lo) > cut) --lo;
            const double f_lo = interp2(cut, lev(lo), lev(lo + 1), freq(lo), freq(lo + 1));
            int64_t hi = i;
            while (hi < n - 1 && lev(hi) > cut) ++hi;
            const double f_hi = interp2(cut, lev(hi - 1), lev(hi), freq(hi - 1), freq(hi));
            o[found] = f_hi - f_lo;
            o[nf + found] = freq(i);
            o[2 * nf + found] = li;
            ++found;
            i = hi;
        } else {
            ++i;
        }
    }
}

}  // namespace

int formants_device(const float* traces, int ntr, int64_t n, double fs, int nf, double* out, cudaStream_t st,
                    std::string* err) {
    const int64_t nh = n / 2 + 1;
    double* x = nullptr;
    double* level = nullptr;
    cufftDoubleComplex* X = nullptr;
    cufftHandle plan = 0;
    bool have_plan = false;
    int status = VS_OK;
    auto fail = [&](int s, const std::string& m) { status = s; *err = m; };
    do {
        if (cudaMalloc(&x, (size_t)ntr * n * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&X, (size_t)ntr * nh * sizeof(cufftDoubleComplex)) != cudaSuccess ||
            cudaMalloc(&level, (size_t)ntr * n * sizeof(double)) != cudaSuccess) {
            fail(VS_ERR_ALLOC, "vs_formants: cudaMalloc failed");
            break;
        }
        const int64_t count = (int64_t)ntr * n;
        to_double_kernel<<<(unsigned)((count + 255) / 256), 256, 0, st>>>(traces, x, count);
        int nn[1] = {(int)n};
        if (cufftPlanMany(&plan, 1, nn, nullptr, 1, (int)n, nullptr, 1, (int)nh, CUFFT_D2Z, ntr) != CUFFT_SUCCESS) {
            fail(VS_ERR_CUDA, "vs_formants: cufftPlanMany failed");
            break;
        }
        have_plan = true;
        if (cufftSetStream(plan, st) != CUFFT_SUCCESS || cufftExecD2Z(plan, x, X) != CUFFT_SUCCESS) {
            fail(VS_ERR_CUDA, "vs_formants: cufftExecD2Z failed");
            break;
        }
        level_kernel<<<(unsigned)((nh * ntr + 255) / 256), 256, 0, st>>>(X, level, n, nh, ntr);
        formant_scan_kernel<<<(ntr + 63) / 64, 64, 0, st>>>(level, n, fs, nf, out, ntr);
        const cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) fail(VS_ERR_CUDA, std::string("vs_formants: ") + cudaGetErrorString(e));
    } while (false);
    if (have_plan) cufftDestroy(plan);
    if (x) cudaFree(x);
    if (X) cudaFree(X);
    if (level) cudaFree(level);
    return status;
}

}  // namespace vsb
