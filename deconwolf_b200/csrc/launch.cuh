// launch.cuh -- launch wrappers for the templated FFT passes.
#pragma once
#include <cuda_runtime.h>
#include <atomic>
#include "passes.cuh"

namespace dwcu {

// Opt a kernel into more than 48 KB of dynamic shared memory, and size a
// persistent grid (resident CTAs per SM x SMs), once per device.
struct KernelOnce {
    std::atomic<unsigned long long> smem_done{0};
    std::atomic<int> grid[64];
    KernelOnce()
    {
        for (auto &g : grid) g.store(0);
    }
};

template <class K>
inline void ensure_smem(KernelOnce &ko, K kernel, size_t bytes)
{
    int dev = 0;
    cudaGetDevice(&dev);
    unsigned long long bit = 1ull << (dev & 63);
    if (bytes > 48 * 1024 && !(ko.smem_done.load() & bit)) {
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) bytes);
        ko.smem_done.fetch_or(bit);
    }
}

template <class K>
inline int persistent_grid(KernelOnce &ko, K kernel, int threads, size_t smem, int ntiles)
{
    int dev = 0;
    cudaGetDevice(&dev);
    int g = ko.grid[dev & 63].load();
    if (g == 0) {
        int per_sm = 0, sms = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        g = (per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
        ko.grid[dev & 63].store(g);
    }
    return ntiles < g ? ntiles : g;
}

template <class RD, int T>
void launch_lines_t(const LinesArgs &a, int nblocks, cudaStream_t st)
{
    static KernelOnce ko, kp;
    using C = LinesCfg<RD, T>;
    constexpr int tpl = C::THREADS / T;
    const size_t smem = a.mode >= LINES_CONV ? C::SMEM_BYTES : C::SMEM_FFT;
    if (a.planes) {
        ensure_smem(kp, k_lines<RD, T, true>, C::SMEM_BYTES);
        k_lines<RD, T, true><<<nblocks, dim3(T, tpl), smem, st>>>(a);
    } else {
        ensure_smem(ko, k_lines<RD, T>, C::SMEM_BYTES);
        k_lines<RD, T><<<nblocks, dim3(T, tpl), smem, st>>>(a);
    }
}

template <class RD, int DIR>
void launch_y_dir(const YArgs &a, cudaStream_t st)
{
    static KernelOnce ko;
    using C = YCfg<RD>;
    ensure_smem(ko, k_ypass<RD, DIR>, C::SMEM_BYTES);
    const int grid = persistent_grid(ko, k_ypass<RD, DIR>, C::THREADS, C::SMEM_BYTES, a.ntiles);
    k_ypass<RD, DIR><<<grid, dim3(C::TX, RD::TPL), C::SMEM_BYTES, st>>>(a);
}

template <class RD>
void launch_y_t(const YArgs &a, cudaStream_t st)
{
    if (a.dir < 0)
        launch_y_dir<RD, -1>(a, st);
    else
        launch_y_dir<RD, +1>(a, st);
}

template <class RD, int R, int FAM>
void launch_x_fam(const XArgs &a, cudaStream_t st)
{
    static KernelOnce ko;
    using C = XCfg<RD, R, FAM>;
    ensure_smem(ko, k_xpass<RD, R, FAM>, C::SMEM_BYTES);
    k_xpass<RD, R, FAM><<<a.ntiles, dim3(C::TPL, C::RY), C::SMEM_BYTES, st>>>(a);
}

// The forward and update families always run over every row; where the
// plan's tiles hold two rows and one row still fills two warps, they run one
// row per CTA (half the shared memory and threads per CTA, twice the CTAs per
// SM to hide each other's barriers).  The ratio and store families keep the
// plan's tiles (the ratio's error partials are counted per plan tile).
template <class RD, int R, int FAM>
void launch_x_rows(const XArgs &a, cudaStream_t st)
{
    constexpr int row_threads = cmax(RD::TPL, RevRad<RD>::TPL);
    if constexpr (R == 2 && row_threads >= 64) {
        XArgs b = a;
        b.ntiles = a.Z * a.Y;
        launch_x_fam<RD, 1, FAM>(b, st);
    } else {
        launch_x_fam<RD, R, FAM>(a, st);
    }
}

// the ops of one SHB / RL iteration (ratio + error, update); an alternate
// radix plan of the autotuner is compiled for these families only
inline bool x_iteration_op(int op)
{
    const int f = x_family(op);
    return f == XFAM_RATIO || f == XFAM_UPDATE;
}

template <class RD, int R>
void launch_x_iter_t(const XArgs &a, cudaStream_t st)
{
    if (x_family(a.op) == XFAM_RATIO)
        launch_x_fam<RD, R, XFAM_RATIO>(a, st);
    else
        launch_x_rows<RD, R, XFAM_UPDATE>(a, st);
}

template <class RD, int R>
void launch_x_t(const XArgs &a, cudaStream_t st)
{
    switch (x_family(a.op)) {
    case XFAM_FWD: launch_x_rows<RD, R, XFAM_FWD>(a, st); break;
    case XFAM_RATIO: launch_x_fam<RD, R, XFAM_RATIO>(a, st); break;
    case XFAM_UPDATE: launch_x_rows<RD, R, XFAM_UPDATE>(a, st); break;
    default: launch_x_fam<RD, R, XFAM_STORE>(a, st); break;
    }
}

}  // namespace dwcu
