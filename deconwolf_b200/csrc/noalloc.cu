// noalloc.cu -- dwcu_fft_r2c_noalloc: the 3-D R2C transform of dwcu_fft_r2c
// without any device-memory allocation.
//
// dwcu_fft_r2c takes its work space with cudaMalloc and returns it with
// cudaFree on every call.  cudaFree synchronises the whole device, so a
// caller that keeps other work in flight on other streams of the same GPU
// (a serving loop that interleaves jobs, a pipeline recording into several
// streams) stalls on every transform, and a caller running under a fixed
// device-memory budget (a memory pool that owns the rest of the GPU) may not
// be able to allocate at all.  This variant uses a fixed work space that is
// part of the library's device image instead: one file-scope array per
// device, looked up once with cudaGetSymbolAddress.
//
// Limits and rules:
//   * the work space holds kScratchBytes (32 MiB); transforms that need more
//     (spectrum + staged input + scalars + twiddle tables, see need_bytes)
//     are rejected with DWCU_ERROR_INVALID_VALUE;
//   * the first call on a device does one-time setup (the symbol lookup,
//     which loads this module, and the kernels' shared-memory attributes),
//     so that first call belongs before any stream capture;
//   * the spectrum, the staged input and the error flags must start at zero:
//     every call clears them on its stream before the transform;
//   * there is one work space per device, so two calls that overlapped on one
//     device would race on it: calls are serialised by a per-device lock and
//     each returns only after its stream has drained.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>

#include "../../include/dwcu.h"
#include "dft.cuh"

namespace dwcu {
struct JobScalars;
int fft3d_scratch_sizes(long long M, long long N, long long P, size_t *spec_bytes, size_t *real_bytes);
int fft3d_r2c_scratch(const float *d_in, long long M, long long N, long long P, float *d_out, cudaStream_t stream,
                      float2 *S, float *real, JobScalars *sc, const float2 *const tw[4]);
void record_error(const char *msg);
void record_launch();
}  // namespace dwcu

namespace {

constexpr size_t kScratchBytes = size_t(32) << 20;
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_mu[kMaxDevices];
void *g_addr[kMaxDevices];  // g_scratch on each device, looked up once

size_t up256(size_t b) { return (b + 255) & ~size_t(255); }

int fail(int code, const char *msg)
{
    dwcu::record_error(msg);
    return code;
}

// restores the caller's current device on every return path
struct DeviceGuard {
    int prev = -1;
    DeviceGuard() { if (cudaGetDevice(&prev) != cudaSuccess) { cudaGetLastError(); prev = -1; } }
    ~DeviceGuard() { if (prev >= 0) cudaSetDevice(prev); }
};

// work already queued on the shared work space must finish before the lock
// is released, whatever went wrong after it was queued
int fail_drained(cudaStream_t st, int code, const char *msg)
{
    cudaStreamSynchronize(st);
    cudaGetLastError();
    return fail(code, msg);
}

// the twiddle table exp(-2 pi i m / n) of the engine (engine.cu computes it
// on the host in double); this file is compiled without FMA contraction, so
// the device evaluates the same double operations and rounds to the same floats
__global__ void k_twiddle_table(float2 *t, long long n)
{
    for (long long m = blockIdx.x * (long long) blockDim.x + threadIdx.x; m < n;
         m += (long long) gridDim.x * blockDim.x)
        t[m] = make_float2((float) dwcu::cx::cospi_frac(2 * m, n), (float) -dwcu::cx::sinpi_frac(2 * m, n));
}

}  // namespace

extern "C" int dwcu_fft_r2c_noalloc(const float *d_in, int64_t M, int64_t N, int64_t P, float *d_out,
                                    int32_t device, void *stream)
{
    if (!d_in || !d_out) return fail(DWCU_ERROR_INVALID_VALUE, "NULL argument");
    if (device < 0 || device >= kMaxDevices) return fail(DWCU_ERROR_INVALID_VALUE, "device out of range");
    size_t spec = 0, real = 0;
    int rc = dwcu::fft3d_scratch_sizes(M, N, P, &spec, &real);
    if (rc) return rc;
    const long long lens[4] = {M, M / 2, N, P};
    size_t need = spec + real + 256;
    for (long long n : lens) need += up256(sizeof(float2) * (size_t) n);
    if (need > kScratchBytes) {
        char msg[200];
        snprintf(msg, sizeof msg,
                 "a %lld x %lld x %lld transform needs %zu bytes of work space; the no-allocation variant has %zu",
                 (long long) M, (long long) N, (long long) P, need, kScratchBytes);
        return fail(DWCU_ERROR_INVALID_VALUE, msg);
    }
    DeviceGuard restore;
    std::lock_guard<std::mutex> lk(g_mu[device]);
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return fail(DWCU_ERROR_CUDA, "cudaSetDevice failed (no usable CUDA device?)");
    }
    if (!g_addr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return fail(DWCU_ERROR_CUDA, "cudaGetSymbolAddress of the work space failed");
        }
        g_addr[device] = p;
    }
    char *base = (char *) g_addr[device];
    cudaStream_t st = stream ? (cudaStream_t) stream : cudaStreamPerThread;
    // spectrum, staged input, scalars: cleared; twiddle tables after them
    if (cudaMemsetAsync(base, 0, spec + real + 256, st) != cudaSuccess)
        return fail_drained(st, DWCU_ERROR_CUDA, "clearing the work space failed");
    const float2 *tw[4];
    size_t off = spec + real + 256;
    for (int i = 0; i < 4; ++i) {
        float2 *t = (float2 *) (base + off);
        const int blocks = (int) ((lens[i] + 255) / 256);
        k_twiddle_table<<<blocks, 256, 0, st>>>(t, lens[i]);
        dwcu::record_launch();
        if (cudaGetLastError() != cudaSuccess) return fail_drained(st, DWCU_ERROR_CUDA, "twiddle launch failed");
        tw[i] = t;
        off += up256(sizeof(float2) * (size_t) lens[i]);
    }
    return dwcu::fft3d_r2c_scratch(d_in, M, N, P, d_out, st, (float2 *) base, (float *) (base + spec),
                                   (dwcu::JobScalars *) (base + spec + real), tw);
}
