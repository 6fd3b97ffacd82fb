// Statically compiled (nvcc, sm_100a) kernels of libsodecl_cuda:
//  * the Euler-Maruyama noise stream, computed by the same device code the
//    NVRTC solver programs embed (device/threefry.cuh), for bit-exactness
//    tests against the CPU generator;
//  * an FMA issue-rate microbenchmark, the denominator of the FP64/FP32
//    "fraction of issue peak" figures;
//  * a check of the reciprocal quotient (device/fastdiv.cuh) against IEEE
//    division on random and special operands.
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "device/fastdiv.cuh"
#include "device/threefry.cuh"
#include "sodecl_cuda.h"

namespace {

__global__ void noise_stream_kernel(const long long *gids, const double *counters, long long n, int nnoi, double dt,
                                    long long nsteps, double *normals, unsigned long long *words, double *u01)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int ncalls = (nnoi + 1) / 2;
    const double sqrt_h = sqrt(dt);
    const unsigned long long gid = (unsigned long long)gids[i];
    double counter = counters[i];
    for (long long s = 0; s < nsteps; ++s) {
        for (int c = 0; c < ncalls; ++c) {
            unsigned long long w0, w1;
            sodecl_threefry2x64_20(gid, sodecl_counter_word(counter), SODECL_TF_KEY0, SODECL_TF_KEY1, w0, w1);
            counter = counter + 1;
            const long long draw = (i * nsteps + s) * ncalls + c;
            if (words) {
                words[2 * draw] = w0;
                words[2 * draw + 1] = w1;
            }
            if (u01) {
                u01[2 * draw] = sodecl_u01_open_open(w0);
                u01[2 * draw + 1] = sodecl_u01_open_open(w1);
            }
            double n0, n1;
            sodecl_gaussian_pair<double>(w0, w1, sqrt_h, n0, n1);
            const long long base = (i * nsteps + s) * nnoi;
            normals[base + 2 * c] = n0;
            if (2 * c + 1 < nnoi) normals[base + 2 * c + 1] = n1;
        }
    }
}

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long &x)
{
    unsigned long long z = (x += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// An operand: mostly random bit patterns over every exponent, some with the
// significand near 1 or 2, some special (0, subnormal, Inf, NaN, extremes).
__device__ __forceinline__ double division_operand(unsigned long long &state)
{
    const unsigned long long u = splitmix64(state);
    const unsigned kind = (unsigned)(u >> 60);
    unsigned long long bits = splitmix64(state);
    if (kind < 8) {
        // exponent within +-600 of 1, where the fast path runs
        const unsigned long long e = 1023 - 600 + (u % 1200);
        bits = (bits & 0x800FFFFFFFFFFFFFULL) | (e << 52);
    } else if (kind < 11) {
        const unsigned long long e = 1023 - 30 + (u % 60);
        const unsigned long long k = (u >> 20) & 63;
        const unsigned long long m = ((u >> 30) & 1) ? k : (0x000FFFFFFFFFFFFFULL - k);
        bits = (bits & 0x8000000000000000ULL) | (e << 52) | m;
    } else if (kind < 15) {
        // anything: full exponent range, subnormals, Inf, NaN
    } else {
        const double special[8] = {0.0, -0.0, 1.0 / 0.0, -1.0 / 0.0, 4.9e-324, 2.2250738585072014e-308,
                                   1.7976931348623157e308, 6.0};
        return special[u & 7];
    }
    return __longlong_as_double((long long)bits);
}

__global__ void division_check_kernel(unsigned long long seed, long long per_thread, unsigned long long *mismatches,
                                      double *first)
{
    unsigned long long state = seed ^ (0xD1B54A32D192ED03ULL * (blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x + 1));
    unsigned long long bad = 0;
    for (long long i = 0; i < per_thread; ++i) {
        const double a = division_operand(state), b = division_operand(state);
        const double want = a / b, got = sodecl_div_rcp(a, b);
        const bool same = (__double_as_longlong(want) == __double_as_longlong(got)) || (want != want && got != got);
        if (!same) {
            if (atomicAdd(mismatches, 1ULL) == 0) {
                first[0] = a;
                first[1] = b;
            }
            ++bad;
        }
    }
    (void)bad;
}

// The same for binary32: random patterns with exponents within +-70 of 1 (the
// fast path and both sides of its bounds), significands near 1 and 2,
// anything, and specials.
__device__ __forceinline__ float division_operand_f32(unsigned long long &state)
{
    const unsigned long long u = splitmix64(state);
    const unsigned kind = (unsigned)(u >> 60);
    unsigned bits = (unsigned)splitmix64(state);
    if (kind < 8) {
        const unsigned e = 127 - 70 + (unsigned)(u % 140);
        bits = (bits & 0x807FFFFFu) | (e << 23);
    } else if (kind < 11) {
        const unsigned e = 127 - 20 + (unsigned)(u % 40);
        const unsigned k = (unsigned)((u >> 20) & 63);
        const unsigned m = ((u >> 30) & 1) ? k : (0x007FFFFFu - k);
        bits = (bits & 0x80000000u) | (e << 23) | m;
    } else if (kind < 15) {
        // anything: full exponent range, subnormals, Inf, NaN
    } else {
        const float special[8] = {0.0f, -0.0f, 1.0f / 0.0f, -1.0f / 0.0f, 1.4e-45f, 1.17549435e-38f, 3.40282347e38f,
                                  6.0f};
        return special[u & 7];
    }
    return __int_as_float((int)bits);
}

__global__ void division_check_f32_kernel(unsigned long long seed, long long per_thread, unsigned long long *mismatches,
                                          float *first)
{
    unsigned long long state = seed ^ (0xD1B54A32D192ED03ULL * (blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x + 1));
    for (long long i = 0; i < per_thread; ++i) {
        const float a = division_operand_f32(state), b = division_operand_f32(state);
        const float want = a / b, got = sodecl_div_rcp(a, b);
        const bool same = (__float_as_int(want) == __float_as_int(got)) || (want != want && got != got);
        if (!same && atomicAdd(mismatches, 1ULL) == 0) {
            first[0] = a;
            first[1] = b;
        }
    }
}

// Eight independent FMA chains per thread, unrolled; every SM full of warps.
template <class T>
__global__ void __launch_bounds__(256) fma_chains_kernel(T *sink, int iters, T a, T b)
{
    T x0 = (T)threadIdx.x * (T)1e-3, x1 = x0 + (T)1, x2 = x0 + (T)2, x3 = x0 + (T)3;
    T x4 = x0 + (T)4, x5 = x0 + (T)5, x6 = x0 + (T)6, x7 = x0 + (T)7;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
            x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
        }
    }
    const T s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
    if (s == (T)-12345.0) sink[blockIdx.x * blockDim.x + threadIdx.x] = s;  // never true; keeps the chains live
}

// Sines at full occupancy: eight independent sums of sin(x_k - y) per thread,
// the coupling term of a Kuramoto row, with arguments within a few units of
// zero (where phases that have drifted apart by a few radians put them).
template <class T>
__global__ void __launch_bounds__(256) sin_sums_kernel(T *sink, int iters, T step)
{
    T x[8], acc[8];
    const T y0 = (T)(threadIdx.x % 64) * (T)0.01;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        x[k] = y0 + (T)k * (T)0.7 - (T)2.5;
        acc[k] = (T)0;
    }
    T y = (T)0;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[k] += sin(x[k] - y);
        y += step;
    }
    const T s = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
    if (s == (T)-12345.0) sink[blockIdx.x * blockDim.x + threadIdx.x] = s;  // never true; keeps the sums live
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) { if (cudaGetDevice(&prev) != cudaSuccess) prev = -1; cudaSetDevice(dev); }
    ~DeviceGuard() { if (prev >= 0) cudaSetDevice(prev); }
};

// The fastest of kTrials timed launches of `launch` (after two warm-up
// launches of `warm`), in ms; err gets the first CUDA error.
template <class Warm, class Launch>
float fastest_launch_ms(Warm warm, Launch launch, cudaError_t *err)
{
    constexpr int kTrials = 7;
    cudaEvent_t e[kTrials + 1];
    for (auto &ev : e) cudaEventCreate(&ev);
    warm();
    launch();
    cudaEventRecord(e[0]);
    for (int k = 0; k < kTrials; ++k) {
        launch();
        cudaEventRecord(e[k + 1]);
    }
    *err = cudaEventSynchronize(e[kTrials]);
    float ms = 0.f;
    for (int k = 0; k < kTrials; ++k) {
        float t = 0.f;
        cudaEventElapsedTime(&t, e[k], e[k + 1]);
        if (k == 0 || t < ms) ms = t;
    }
    for (auto &ev : e) cudaEventDestroy(ev);
    return ms;
}

template <class T>
int run_fma_peak(int device, double *fma_per_s, double *ms_out)
{
    DeviceGuard guard(device);
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) { cudaGetLastError(); return SODECL_ERR_NO_DEVICE; }
    const int block = 256;
    const int blocks = prop.multiProcessorCount * 8;
    const int iters = 1 << 15;
    T *sink = nullptr;
    if (cudaMalloc(&sink, sizeof(T) * (size_t)blocks * block) != cudaSuccess) { cudaGetLastError(); return SODECL_ERR_OUT_OF_MEMORY; }
    const T a = (T)0.999999, b = (T)1e-7;
    // the fastest of 7 timed launches (about 20 ms each for FP64)
    cudaError_t err = cudaSuccess;
    const float ms = fastest_launch_ms([&] { fma_chains_kernel<T><<<blocks, block>>>(sink, iters / 8, a, b); },
                                       [&] { fma_chains_kernel<T><<<blocks, block>>>(sink, iters, a, b); }, &err);
    cudaFree(sink);
    if (err != cudaSuccess) { cudaGetLastError(); return SODECL_ERR_CUDA; }
    const double fmas = (double)blocks * block * (double)iters * 4.0 * 8.0;
    if (fma_per_s) *fma_per_s = fmas / (ms * 1e-3);
    if (ms_out) *ms_out = ms;
    return SODECL_OK;
}

template <class T>
int run_sin_peak(int device, double *sin_per_s, double *ms_out)
{
    DeviceGuard guard(device);
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) { cudaGetLastError(); return SODECL_ERR_NO_DEVICE; }
    const int block = 256;
    const int blocks = prop.multiProcessorCount * 8;
    const int iters = 2048;  // about 20 ms a launch in FP64
    T *sink = nullptr;
    if (cudaMalloc(&sink, sizeof(T) * (size_t)blocks * block) != cudaSuccess) { cudaGetLastError(); return SODECL_ERR_OUT_OF_MEMORY; }
    const T step = (T)2e-3;
    cudaError_t err = cudaSuccess;
    const float ms = fastest_launch_ms([&] { sin_sums_kernel<T><<<blocks, block>>>(sink, iters / 8, step); },
                                       [&] { sin_sums_kernel<T><<<blocks, block>>>(sink, iters, step); }, &err);
    cudaFree(sink);
    if (err != cudaSuccess) { cudaGetLastError(); return SODECL_ERR_CUDA; }
    const double sines = (double)blocks * block * (double)iters * 8.0;
    if (sin_per_s) *sin_per_s = sines / (ms * 1e-3);
    if (ms_out) *ms_out = ms;
    return SODECL_OK;
}

}  // namespace

extern "C" int sodecl_cuda_noise_stream(int device, const int64_t *gids, const double *counters, int64_t n, int32_t nnoi,
                                        double dt_program, int64_t nsteps, double *normals, uint64_t *words, double *u01)
{
    if (!gids || !counters || !normals || n < 1 || nnoi < 1 || nsteps < 1 || !(dt_program > 0)) return SODECL_ERR_INVALID_ARG;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) { cudaGetLastError(); return SODECL_ERR_NO_DEVICE; }
    DeviceGuard guard(device);
    const int ncalls = (nnoi + 1) / 2;
    const size_t n_norm = (size_t)n * nsteps * nnoi, n_draw = (size_t)n * nsteps * ncalls * 2;
    long long *d_gid = nullptr;
    double *d_cnt = nullptr, *d_norm = nullptr, *d_u01 = nullptr;
    unsigned long long *d_words = nullptr;
    int rc = SODECL_OK;
    auto check = [&](cudaError_t e) { if (e != cudaSuccess && rc == SODECL_OK) { rc = (e == cudaErrorMemoryAllocation) ? SODECL_ERR_OUT_OF_MEMORY : SODECL_ERR_CUDA; cudaGetLastError(); } };
    check(cudaMalloc(&d_gid, n * sizeof(long long)));
    check(cudaMalloc(&d_cnt, n * sizeof(double)));
    check(cudaMalloc(&d_norm, n_norm * sizeof(double)));
    if (words) check(cudaMalloc(&d_words, n_draw * sizeof(unsigned long long)));
    if (u01) check(cudaMalloc(&d_u01, n_draw * sizeof(double)));
    if (rc == SODECL_OK) {
        check(cudaMemcpy(d_gid, gids, n * sizeof(long long), cudaMemcpyHostToDevice));
        check(cudaMemcpy(d_cnt, counters, n * sizeof(double), cudaMemcpyHostToDevice));
    }
    if (rc == SODECL_OK) {
        const int block = 128;
        noise_stream_kernel<<<(unsigned)((n + block - 1) / block), block>>>(d_gid, d_cnt, n, nnoi, dt_program, nsteps, d_norm, d_words, d_u01);
        check(cudaGetLastError());
        check(cudaDeviceSynchronize());
    }
    if (rc == SODECL_OK) {
        check(cudaMemcpy(normals, d_norm, n_norm * sizeof(double), cudaMemcpyDeviceToHost));
        if (words) check(cudaMemcpy(words, d_words, n_draw * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
        if (u01) check(cudaMemcpy(u01, d_u01, n_draw * sizeof(double), cudaMemcpyDeviceToHost));
    }
    cudaFree(d_gid);
    cudaFree(d_cnt);
    cudaFree(d_norm);
    cudaFree(d_words);
    cudaFree(d_u01);
    return rc;
}

extern "C" int sodecl_cuda_division_check(int device, int64_t pairs, uint64_t seed, int64_t *mismatches,
                                          double *first_a, double *first_b)
{
    if (pairs < 1 || !mismatches) return SODECL_ERR_INVALID_ARG;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) { cudaGetLastError(); return SODECL_ERR_NO_DEVICE; }
    DeviceGuard guard(device);
    const int block = 256, blocks = 148 * 8;
    const long long per_thread = (pairs + (long long)block * blocks - 1) / ((long long)block * blocks);
    unsigned long long *d_bad = nullptr;
    double *d_first = nullptr;
    if (cudaMalloc(&d_bad, sizeof(unsigned long long)) != cudaSuccess ||
        cudaMalloc(&d_first, 2 * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(d_bad);
        return SODECL_ERR_OUT_OF_MEMORY;
    }
    int rc = SODECL_OK;
    cudaMemset(d_bad, 0, sizeof(unsigned long long));
    cudaMemset(d_first, 0, 2 * sizeof(double));
    division_check_kernel<<<blocks, block>>>(seed, per_thread, d_bad, d_first);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) rc = SODECL_ERR_CUDA;
    unsigned long long bad = 0;
    double first[2] = {0.0, 0.0};
    if (rc == SODECL_OK) {
        cudaMemcpy(&bad, d_bad, sizeof(bad), cudaMemcpyDeviceToHost);
        cudaMemcpy(first, d_first, sizeof(first), cudaMemcpyDeviceToHost);
    }
    cudaFree(d_bad);
    cudaFree(d_first);
    *mismatches = (int64_t)bad;
    if (first_a) *first_a = first[0];
    if (first_b) *first_b = first[1];
    return rc;
}

extern "C" int sodecl_cuda_division_check_f32(int device, int64_t pairs, uint64_t seed, int64_t *mismatches,
                                              float *first_a, float *first_b)
{
    if (pairs < 1 || !mismatches) return SODECL_ERR_INVALID_ARG;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) { cudaGetLastError(); return SODECL_ERR_NO_DEVICE; }
    DeviceGuard guard(device);
    const int block = 256, blocks = 148 * 8;
    const long long per_thread = (pairs + (long long)block * blocks - 1) / ((long long)block * blocks);
    unsigned long long *d_bad = nullptr;
    float *d_first = nullptr;
    if (cudaMalloc(&d_bad, sizeof(unsigned long long)) != cudaSuccess ||
        cudaMalloc(&d_first, 2 * sizeof(float)) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(d_bad);
        return SODECL_ERR_OUT_OF_MEMORY;
    }
    int rc = SODECL_OK;
    cudaMemset(d_bad, 0, sizeof(unsigned long long));
    cudaMemset(d_first, 0, 2 * sizeof(float));
    division_check_f32_kernel<<<blocks, block>>>(seed, per_thread, d_bad, d_first);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) rc = SODECL_ERR_CUDA;
    unsigned long long bad = 0;
    float first[2] = {0.0f, 0.0f};
    if (rc == SODECL_OK) {
        cudaMemcpy(&bad, d_bad, sizeof(bad), cudaMemcpyDeviceToHost);
        cudaMemcpy(first, d_first, sizeof(first), cudaMemcpyDeviceToHost);
    }
    cudaFree(d_bad);
    cudaFree(d_first);
    *mismatches = (int64_t)bad;
    if (first_a) *first_a = first[0];
    if (first_b) *first_b = first[1];
    return rc;
}

extern "C" int sodecl_cuda_fma_peak(int device, int32_t precision, double *fma_per_s, double *ms)
{
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) { cudaGetLastError(); return SODECL_ERR_NO_DEVICE; }
    if (precision == SODECL_FP64) return run_fma_peak<double>(device, fma_per_s, ms);
    if (precision == SODECL_FP32) return run_fma_peak<float>(device, fma_per_s, ms);
    return SODECL_ERR_INVALID_ARG;
}

extern "C" int sodecl_cuda_sin_peak(int device, int32_t precision, double *sin_per_s, double *ms)
{
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) { cudaGetLastError(); return SODECL_ERR_NO_DEVICE; }
    if (precision == SODECL_FP64) return run_sin_peak<double>(device, sin_per_s, ms);
    if (precision == SODECL_FP32) return run_sin_peak<float>(device, sin_per_s, ms);
    return SODECL_ERR_INVALID_ARG;
}
