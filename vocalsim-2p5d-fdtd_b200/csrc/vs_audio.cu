// vs_audio.cu -- WAV samples of listener traces on the device.
//
// Restates results/generate_audio.py:14-42 of the reference for a batch of
// traces: audio = P / max|P| clipped to [-1, 1]; for srate_mul > 1 a
// 2nd-order Butterworth low-pass at 5050 Hz (scipy.signal.butter(2, Wn)
// with Wn = 5050 / (44100 srate_mul / 2)) applied as scipy.signal.lfilter
// applies it -- the direct form II transposed recursion in double,
//   y = b0 x + z0;  z0 = (z1 + x b1) - y a1;  z1 = x b2 - y a2,
// zero initial state -- and every srate_mul-th sample kept (filtered[::mul]);
// the samples are rounded to float32 as the WAV is written.  One block per
// trace: the block reduces max|P|, one thread then runs the recursion (it
// is sequential by definition) and writes the kept samples.
#include <cuda_runtime.h>

#include <cmath>
#include <complex>
#include <string>

#include "vs_device.h"

namespace vsb {
namespace {

constexpr double kAudioCutoffHz = 5050.0;   // generate_audio.py:29
constexpr int kAudioThreads = 256;

__global__ void audio_kernel(const float* __restrict__ traces, int64_t n, int mul, double b0, double b1, double b2,
                             double a1, double a2, float* __restrict__ out, int64_t nout) {
    const float* x = traces + (int64_t)blockIdx.x * n;
    float* y = out + (int64_t)blockIdx.x * nout;
    __shared__ float red[kAudioThreads];
    float m = 0.0f;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) m = fmaxf(m, fabsf(x[i]));
    red[threadIdx.x] = m;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) red[threadIdx.x] = fmaxf(red[threadIdx.x], red[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    const double maxp = (double)red[0];
    double z0 = 0.0, z1 = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        double a = __ddiv_rn((double)x[i], maxp);
        a = a < -1.0 ? -1.0 : (a > 1.0 ? 1.0 : a);     // numpy.clip: NaN stays NaN
        if (mul == 1) {
            y[i] = (float)a;
            continue;
        }
        const double yi = __dadd_rn(z0, __dmul_rn(b0, a));
        z0 = __dsub_rn(__dadd_rn(z1, __dmul_rn(a, b1)), __dmul_rn(yi, a1));
        z1 = __dsub_rn(__dmul_rn(a, b2), __dmul_rn(yi, a2));
        if (i % mul == 0) y[i / mul] = (float)yi;
    }
}

}  // namespace

// butter(2, Wn, 'low') as scipy.signal designs it: analog prototype poles
// -exp(i pi m / 4), m = -1, 1; pre-warp w = 2 fs tan(pi Wn / fs) with fs = 2;
// poles times w, gain w^2; bilinear transform (fs2 = 2 fs): poles
// (fs2 + p) / (fs2 - p), two zeros at -1, gain k / prod(fs2 - p);
// b = k [1, 2, 1], a = real(poly(poles)).
void audio_filter(int srate_mul, double b[3], double a[3]) {
    const double pi = 3.14159265358979323846;
    const double wn = kAudioCutoffHz / (44100.0 * srate_mul / 2.0);
    const double fs = 2.0, fs2 = 2.0 * fs;
    const double warped = 2.0 * fs * std::tan(pi * wn / fs);
    std::complex<double> p[2];
    for (int i = 0; i < 2; ++i) {
        const double m = i == 0 ? -1.0 : 1.0;
        p[i] = -std::exp(std::complex<double>(0.0, pi * m / 4.0)) * warped;
    }
    const double k = warped * warped;
    const std::complex<double> z0 = (fs2 + p[0]) / (fs2 - p[0]), z1 = (fs2 + p[1]) / (fs2 - p[1]);
    const double kz = k * (1.0 / ((fs2 - p[0]) * (fs2 - p[1]))).real();
    b[0] = kz; b[1] = 2.0 * kz; b[2] = kz;
    a[0] = 1.0;
    a[1] = (-(z0 + z1)).real();
    a[2] = (z0 * z1).real();
}

int audio_device(const float* traces, int ntr, int64_t n, int mul, float* out, cudaStream_t st, std::string* err) {
    double b[3], a[3];
    audio_filter(mul, b, a);
    const int64_t nout = (n + mul - 1) / mul;
    audio_kernel<<<ntr, kAudioThreads, 0, st>>>(traces, n, mul, b[0], b[1], b[2], a[1], a[2], out, nout);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        *err = std::string("vs_audio: ") + cudaGetErrorString(e);
        return VS_ERR_CUDA;
    }
    return VS_OK;
}

}  // namespace vsb
