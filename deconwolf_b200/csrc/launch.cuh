// launch.cuh -- launch wrappers for the templated FFT passes.
#pragma once
#include <cuda_runtime.h>
#include <atomic>
#include "passes.cuh"

namespace dwcu {

// Opt a kernel into more than 48 KB of dynamic shared memory once per device.
template <class K>
inline void ensure_smem(K kernel, size_t bytes)
{
    static std::atomic<unsigned long long> done{0};
    int dev = 0;
    cudaGetDevice(&dev);
    unsigned long long bit = 1ull << (dev & 63);
    if (bytes > 48 * 1024 && !(done.load() & bit)) {
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) bytes);
        done.fetch_or(bit);
    }
}

template <class RD, int T>
void launch_lines_t(const LinesArgs &a, int nblocks, cudaStream_t st)
{
    using C = LinesCfg<RD, T>;
    ensure_smem(k_lines<RD, T>, C::SMEM_BYTES);
    constexpr int tpl = C::THREADS / T;
    k_lines<RD, T><<<nblocks, dim3(T, tpl), C::SMEM_BYTES, st>>>(a);
}

template <class RD, int R>
void launch_x_t(const XArgs &a, int nblocks, cudaStream_t st)
{
    using C = XCfg<RD, R>;
    ensure_smem(k_xpass<RD, R>, C::SMEM_BYTES);
    k_xpass<RD, R><<<nblocks, dim3(C::TPL, R), C::SMEM_BYTES, st>>>(a);
}

}  // namespace dwcu
