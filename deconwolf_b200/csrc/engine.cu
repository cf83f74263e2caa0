// engine.cu -- host side of the engine: plans, jobs, iteration schedule, C ABI.
//
// One job = one image deconvolution with all of its state resident in HBM:
//   g    image (pitched rows)                G bytes
//   S    working half-spectrum                C bytes
//   K    OTF (scaled by 1/(X*Y*Z))            C bytes
//   xa   estimate x_k                         R bytes
//   xb   previous estimate x_{k-1} (SHB)      R bytes
//   W    Bertero weights (bq > 0)             R bytes
// plus the per-iteration error partials and trace.  One SHB iteration is
//   y-fwd, z-conv(K), y-inv, x[C2R -> I-div -> ratio -> R2C],
//   y-fwd, z-conv(conj K), y-inv, x[C2R -> update -> next extrapolation -> R2C]
// i.e. 8 passes over the spectrum and one read/write of the estimates.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>  // header-only: ranges cost a pointer test unless a tool is attached

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/dwcu.h"
#include "misc_kernels.cuh"
#include "plans_gen.h"

namespace dwcu {

// ------------------------------------------------------------ errors

static thread_local std::string g_last_error;
static thread_local long long g_launches = 0;

static int fail(int code, const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

// for the library's other translation units (host.cu)
void record_error(const char *msg) { g_last_error = msg; }
void record_launch() { ++g_launches; }

#define CU(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return fail(e_ == cudaErrorMemoryAllocation ? DWCU_ERROR_OUT_OF_MEMORY : DWCU_ERROR_CUDA, \
                        "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

#define CHECK_LAUNCH()                                                                        \
    do {                                                                                      \
        ++g_launches;                                                                         \
        cudaError_t e_ = cudaGetLastError();                                                  \
        if (e_ != cudaSuccess)                                                                \
            return fail(DWCU_ERROR_CUDA, "kernel launch failed: %s (%s:%d)", cudaGetErrorString(e_), \
                        __FILE__, __LINE__);                                                  \
    } while (0)

// ------------------------------------------------------------ profiling

struct ProfRec {
    int cls;
    cudaEvent_t a, b;
    bool owned_by_graph;  // events live in a cached graph: never returned to the pool
};
struct ProfClass {
    std::string name;
    double bytes;
};
static std::mutex g_prof_mu;
static bool g_prof_on = false;
static thread_local bool g_tuning = false;  // the autotuner's launches are not profiled
static std::vector<ProfRec> g_prof_recs;
static std::vector<cudaEvent_t> g_prof_pool;
static std::vector<ProfClass> g_prof_classes;

static int prof_class(const char *name, double bytes)
{
    for (size_t i = 0; i < g_prof_classes.size(); ++i)
        if (g_prof_classes[i].name == name && g_prof_classes[i].bytes == bytes) return (int) i;
    g_prof_classes.push_back({name, bytes});
    return (int) g_prof_classes.size() - 1;
}

static cudaEvent_t prof_event()
{
    if (!g_prof_pool.empty()) {
        cudaEvent_t e = g_prof_pool.back();
        g_prof_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// bracket one launch (the scope's lifetime): CUDA-event timing of the
// launch's kernel class when profiling is on, and an NVTX range with the
// class name for trace tools (nsys, ncu --nvtx)
struct ProfScope {
    bool on = false;
    ProfRec rec{};
    cudaStream_t st = nullptr;
    ProfScope(const char *name, double bytes, cudaStream_t s)
    {
        nvtxRangePushA(name);
        std::lock_guard<std::mutex> lk(g_prof_mu);
        if (!g_prof_on || g_tuning) return;
        on = true;
        st = s;
        rec.cls = prof_class(name, bytes);
        rec.a = prof_event();
        rec.b = prof_event();
        rec.owned_by_graph = capturing(s);
        // inside stream capture a plain record is only a dependency edge;
        // the external flag makes it a timing node of the graph
        cudaEventRecordWithFlags(rec.a, st, capturing(st) ? cudaEventRecordExternal : 0);
    }
    static bool capturing(cudaStream_t s)
    {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        return cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusActive;
    }
    ~ProfScope()
    {
        nvtxRangePop();
        if (!on) return;
        cudaEventRecordWithFlags(rec.b, st, capturing(st) ? cudaEventRecordExternal : 0);
        std::lock_guard<std::mutex> lk(g_prof_mu);
        g_prof_recs.push_back(rec);
    }
};

// an NVTX range over one phase of a job (set-up, iterations, result)
struct PhaseRange {
    explicit PhaseRange(const char *name) { nvtxRangePushA(name); }
    ~PhaseRange() { nvtxRangePop(); }
};

// ------------------------------------------------------------ plans

static const LinesPlan *find_lines(int n)
{
    for (const auto &p : kLinesPlans)
        if (p.n == n) return &p;
    return nullptr;
}
static const XPlan *find_x(int n)
{
    for (const auto &p : kXPlans)
        if (p.n == n) return &p;
    return nullptr;
}

// smallest supported length >= w (exact: only w itself)
static long long pad_lines(long long w, bool exact)
{
    if (w == 1) return 1;
    if (exact) return find_lines((int) w) ? w : -1;
    for (const auto &p : kLinesPlans)
        if (p.n >= w) return p.n;
    return -1;
}
static long long pad_x(long long w, bool exact)
{
    // X even with X/2 supported by the x pass
    if (exact) return (w % 2 == 0 && find_x((int) (w / 2))) ? w : -1;
    for (const auto &p : kXPlans)
        if (2LL * p.n >= w) return 2LL * p.n;
    return -1;
}

struct Geometry {
    long long M, N, P, pM, pN, pP;
    long long wM, wN, wP;   // the reference's job size (method_shb.c:137-153)
    long long X, Y, Z;      // padded job size
    long long XP;           // real row pitch (X rounded up to a multiple of 4)
    long long NKB;          // kx blocks of the spectrum layout (X/2+1 over KB)
    long long GP;           // image row pitch (multiple of 4)
    const XPlan *xp;
    const LinesPlan *yp, *zp;
    const YPlan *ytp;       // pipelined y pass when the tile fits shared memory
    // Periodic axes: with border_quality 0 or 1 the reference convolves
    // circularly with period w.  An axis whose exact length w has no
    // supported transform is transformed at a length >= w + 2h instead: the
    // fields live on [0, w), the margins [w, w+h) and [len-h, len) hold
    // copies of [0, h) and [w-h, w), so the linear convolution by the PSF
    // (half-width h about its centre) equals the circular one on [0, w).
    bool wx = false, wy = false, wz = false;
    long long hx = 0, hy = 0, hz = 0;
    long long spec_elems() const { return Z * NKB * Y * KB; }
    long long real_elems() const { return XP * Y * Z; }
};

static const YPlan *find_y(int n)
{
    for (const auto &p : kYPlans)
        if (p.n == n) return &p;
    return nullptr;
}

// candidate `cand` of a length (find_*: candidate 0, listed first)
static const LinesPlan *lines_plan(int n, int cand)
{
    for (const auto &p : kLinesPlans)
        if (p.n == n && p.cand == cand) return &p;
    return nullptr;
}
static const XPlan *x_plan(int n, int cand)
{
    for (const auto &p : kXPlans)
        if (p.n == n && p.cand == cand) return &p;
    return nullptr;
}
static const YPlan *y_plan(int n, int cand)
{
    for (const auto &p : kYPlans)
        if (p.n == n && p.cand == cand) return &p;
    return nullptr;
}

// the autotuner's table (tune.cu)
int tune_plan_count(int kind, int n);
int tune_mode();
float tune_margin();
int tune_lookup(int device, int kind, int n);
void tune_record(int device, int kind, int n, const std::vector<float> &ms, int cand);
int tune_select_idx(const float *ms, int n, float margin);

static int make_geometry(long long M, long long N, long long P, long long pM, long long pN, long long pP, int bq,
                         Geometry &g)
{
    if (M < 1 || N < 1 || P < 1 || pM < 1 || pN < 1 || pP < 1)
        return fail(DWCU_ERROR_INVALID_VALUE, "image and PSF sizes must be positive");
    g.M = M; g.N = N; g.P = P; g.pM = pM; g.pN = pN; g.pP = pP;
    if (bq == 2) {
        g.wM = M + pM - 1; g.wN = N + pN - 1; g.wP = P + pP - 1;
    } else if (bq == 1) {
        g.wM = M + (pM + 1) / 2; g.wN = N + (pN + 1) / 2; g.wP = P + (pP + 1) / 2;
    } else if (bq == 0) {
        g.wM = std::max(M, pM); g.wN = std::max(N, pN); g.wP = std::max(P, pP);
    } else {
        return fail(DWCU_ERROR_INVALID_VALUE, "border_quality must be 0, 1 or 2 (got %d)", bq);
    }
    // Only bq = 2 leaves room for the whole PSF around the image, so only then
    // is a larger (padded) transform size mathematically identical to the
    // reference's job size; bq 0 and 1 wrap around and need the exact size.
    const bool exact = (bq != 2);
    g.X = pad_x(g.wM, exact);
    g.Y = pad_lines(g.wN, exact);
    g.Z = pad_lines(g.wP, exact);
    if (exact) {
        // axes without a transform of the exact length: periodic margins
        if (g.X < 0) { g.wx = true; g.hx = (pM - 1) / 2; g.X = pad_x(g.wM + 2 * g.hx, false); }
        if (g.Y < 0) { g.wy = true; g.hy = (pN - 1) / 2; g.Y = pad_lines(g.wN + 2 * g.hy, false); }
        if (g.Z < 0) { g.wz = true; g.hz = (pP - 1) / 2; g.Z = pad_lines(g.wP + 2 * g.hz, false); }
    }
    if (g.X < 0 || g.Y < 0 || g.Z < 0)
        return fail(DWCU_ERROR_UNSUPPORTED, "no supported FFT size for job %lld x %lld x %lld (border_quality %d)",
                    g.wM, g.wN, g.wP, bq);
    g.xp = find_x((int) (g.X / 2));
    g.yp = g.Y > 1 ? find_lines((int) g.Y) : nullptr;
    g.zp = find_lines((int) g.Z);  // also for Z == 1: the z pass carries the OTF multiply
    if (!g.xp || !g.zp) return fail(DWCU_ERROR_UNSUPPORTED, "x length %lld or z length %lld unsupported", g.X, g.Z);
    g.XP = (g.X + 3) & ~3LL;
    g.NKB = (g.X / 2 + 1 + KB - 1) / KB;
    g.GP = (M + 3) & ~3LL;
    g.ytp = g.Y > 1 ? find_y((int) g.Y) : nullptr;
    return DWCU_SUCCESS;
}

// x-pass tiles (= error partials): R rows of one z plane
static long long x_blocks(const Geometry &g) { return g.Z * ((g.Y + g.xp->R - 1) / g.xp->R); }

// ------------------------------------------------------------ twiddles

struct DeviceCtx {
    int device = -1;
    cudaStream_t stream = nullptr;
    cudaStream_t copy = nullptr;  // image uploads that overlap a job's set-up passes
    std::map<long long, float2 *> tw;  // length -> exp(-2 pi i m / length)
};

static std::mutex g_ctx_mu;
static std::map<int, DeviceCtx *> g_ctx;

static int get_ctx(int device, DeviceCtx **out)
{
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    auto it = g_ctx.find(device);
    if (it != g_ctx.end()) {
        *out = it->second;
        return DWCU_SUCCESS;
    }
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return fail(DWCU_ERROR_CUDA, "no CUDA device available (the engine has no CPU path)");
    }
    if (device < 0 || device >= n) return fail(DWCU_ERROR_INVALID_VALUE, "device %d out of range (%d)", device, n);
    CU(cudaSetDevice(device));
    auto *c = new DeviceCtx();
    c->device = device;
    CU(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    CU(cudaStreamCreateWithFlags(&c->copy, cudaStreamNonBlocking));
    g_ctx[device] = c;
    *out = c;
    return DWCU_SUCCESS;
}

// gaussian_kernel (fim.c:2077-2106): 2*ceil(3 sigma)+1 taps with the
// reference's mixed float/double arithmetic, normalised to sum 1
static GaussTaps gauss_taps(float sigma)
{
    GaussTaps K{};
    int len = (int) std::ceil(3.0 * sigma);
    if (len < 1) len = 1;
    const int n = 2 * len + 1;
    K.n = n;
    const float mid = (n - 1) / 2;
    const float s2 = (float) std::pow((double) sigma, 2.0);
    const float k0 = (float) (1.0 / sigma / std::sqrt(2.0 * M_PI));
    double sum = 0;
    for (int kk = 0; kk < n; ++kk) {
        const float x = (float) kk - mid;
        K.k[kk] = (float) ((double) k0 * std::exp(-0.5 * std::pow((double) x, 2.0) / (double) s2));
        sum += K.k[kk];
    }
    for (int kk = 0; kk < n; ++kk) K.k[kk] = (float) ((double) K.k[kk] / sum);
    return K;
}

// twiddle table of a length, evaluated in double from the exact angle
// reduction in dft.cuh and rounded once to float
static int get_twiddles(DeviceCtx *c, long long n, const float2 **out)
{
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    auto it = c->tw.find(n);
    if (it != c->tw.end()) {
        *out = it->second;
        return DWCU_SUCCESS;
    }
    std::vector<float2> h((size_t) n);
    for (long long m = 0; m < n; ++m)
        h[(size_t) m] = make_float2((float) cx::cospi_frac(2 * m, n), (float) -cx::sinpi_frac(2 * m, n));
    float2 *d = nullptr;
    CU(cudaMalloc(&d, sizeof(float2) * (size_t) n));
    CU(cudaMemcpy(d, h.data(), sizeof(float2) * (size_t) n, cudaMemcpyHostToDevice));
    c->tw[n] = d;
    *out = d;
    return DWCU_SUCCESS;
}

// ------------------------------------------------------------ memory blocks
//
// A job's device memory is one block.  Released blocks are kept per device
// (a few at most) and handed to the next job that fits and needs at least
// four fifths of the block, so a stream of similar-sized jobs (tiles,
// repeated deconvolutions) allocates once; the iteration graphs captured on
// a block stay valid with it and are reused.

struct Block {
    char *ptr = nullptr;
    size_t bytes = 0;
    int device = 0;
    struct Graph {
        cudaGraphExec_t exec = nullptr;
        long long kernels = 0;
        std::vector<ProfRec> recs;  // timing events recorded by the graph's nodes
    };
    std::map<std::string, Graph> graphs;
};

static std::mutex g_blk_mu;
static std::map<int, std::vector<Block *>> g_blk_free;
// released blocks kept per device: at most this many, and at most half of
// the device's memory together
constexpr size_t kMaxCachedBlocks = 64;

static size_t device_total_bytes(int device)
{
    static std::mutex mu;
    static std::map<int, size_t> total;
    std::lock_guard<std::mutex> lk(mu);
    auto it = total.find(device);
    if (it != total.end()) return it->second;
    cudaDeviceProp prop;
    size_t t = cudaGetDeviceProperties(&prop, device) == cudaSuccess ? prop.totalGlobalMem : 0;
    cudaGetLastError();
    total[device] = t;
    return t;
}

static bool trace_on()
{
    static int on = -1;
    if (on < 0) {
        const char *e = getenv("DWCU_TRACE");
        on = (e && *e && *e != '0') ? 1 : 0;
    }
    return on == 1;
}

static void block_free(Block *b)
{
    if (!b) return;
    for (auto &kv : b->graphs) {
        cudaGraphExecDestroy(kv.second.exec);
        for (auto &r : kv.second.recs) {
            cudaEventDestroy(r.a);
            cudaEventDestroy(r.b);
        }
    }
    if (b->ptr) cudaFree(b->ptr);
    delete b;
}

static Block *block_get(int device, size_t bytes)
{
    {
        std::lock_guard<std::mutex> lk(g_blk_mu);
        // the smallest cached block that holds the job and wastes at most a
        // fifth of itself (tiles of a few neighbouring sizes share blocks)
        auto &v = g_blk_free[device];
        size_t best = v.size();
        for (size_t i = 0; i < v.size(); ++i)
            if (v[i]->bytes >= bytes && (double) v[i]->bytes <= 1.25 * (double) bytes &&
                (best == v.size() || v[i]->bytes < v[best]->bytes))
                best = i;
        if (best < v.size()) {
            Block *b = v[best];
            v.erase(v.begin() + (long) best);
            return b;
        }
    }
    Block *b = new Block();
    b->bytes = bytes;
    b->device = device;
    cudaError_t e = cudaMalloc(&b->ptr, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        // release the cached blocks of this device and retry once
        std::vector<Block *> drop;
        {
            std::lock_guard<std::mutex> lk(g_blk_mu);
            drop.swap(g_blk_free[device]);
        }
        for (auto *d : drop) block_free(d);
        e = cudaMalloc(&b->ptr, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            delete b;
            return nullptr;
        }
    }
    return b;
}

static void block_put(Block *b)
{
    if (!b) return;
    std::vector<Block *> drop;
    {
        std::lock_guard<std::mutex> lk(g_blk_mu);
        auto &v = g_blk_free[b->device];
        v.push_back(b);
        const double cap = 0.5 * (double) device_total_bytes(b->device);
        double held = 0;
        for (auto *c : v) held += (double) c->bytes;
        while (!v.empty() && (v.size() > kMaxCachedBlocks || held > cap)) {
            held -= (double) v.front()->bytes;
            drop.push_back(v.front());
            v.erase(v.begin());
        }
    }
    for (auto *d : drop) block_free(d);
}

// ------------------------------------------------------------ host iterator

// dw_iterator_t and dw_iterator_{new,next,set_error} (src/dw.h:298-306,
// src/dw.c:219-276)
struct Iter {
    float error = 1, lasterror = 1;
    int iter = -1, niter = 0;
    float relerror = 0, abserror = 0;
    int itertype = DWCU_ITER_FIXED;
    void init(const dwcu_opts &s)
    {
        error = 1; lasterror = 1;
        itertype = s.iter_type;
        abserror = s.err_abs;
        relerror = s.err_rel;
        iter = -1;
        niter = (s.iter_type != DWCU_ITER_FIXED) ? s.maxiter : s.n_iter;
    }
    int next()
    {
        iter++;
        if (itertype == DWCU_ITER_REL) {
            if (iter < 2) lasterror = 2 * error * relerror;
            if (std::fabs(error - lasterror) / error < relerror) return -1;
        } else if (itertype == DWCU_ITER_ABS) {
            if (iter > 0 && error < abserror) return -1;
        }
        if (iter >= niter) return -1;
        return iter;
    }
    void set(float e)
    {
        lasterror = error;
        error = e;
    }
};

// ------------------------------------------------------------ the job

static inline size_t align256(size_t v) { return (v + 255) & ~(size_t) 255; }

}  // namespace dwcu

struct dwcu_job {
    dwcu_opts s;
    dwcu::Geometry g;
    dwcu::DeviceCtx *ctx = nullptr;
    cudaStream_t stream = nullptr;
    // device memory
    dwcu::Block *block = nullptr;
    char *base = nullptr;
    size_t bytes = 0;
    float *gimg = nullptr;
    float2 *S = nullptr, *K = nullptr;
    float *xa = nullptr, *xb = nullptr, *W = nullptr;
    double *partial = nullptr;
    dwcu::JobScalars *sc = nullptr;
    float *err = nullptr;          // device error trace
    long long *amax = nullptr;
    dwcu::StatsPartial *spart = nullptr;
    dwcu::ArgmaxPartial *apart = nullptr;
    float *psf_dev = nullptr;      // staging for the PSF
    int n_spart = 0, n_apart = 0;
    long long nxb = 0;             // x-pass blocks (= error partials)
    const float2 *tw_x = nullptr, *tw_l = nullptr, *tw_y = nullptr, *tw_z = nullptr;
    // iteration state
    dwcu::Iter it;
    int k_next = -1;               // iteration whose forward half runs next; -1: finished
    bool spectrum_ready = false;   // S holds the transform of iteration k_next's input
    int done_iters = 0;
    bool finished = false;
    bool setup_done = false;
    std::vector<float> trace;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
    bool loop_started = false;
    cudaGraphExec_t graph = nullptr; // a graph owned by this job (holding timing events)
    double enqueue_s = 0;          // host time inside job_step
    std::vector<size_t> guards;    // offsets of the guard bands in the block (debug mode)
    // a part of an image split over GPUs by z planes: the OTF of the part's
    // z-pass columns (all Z planes) takes the place of the spectrum-sized
    // OTF, and T holds the columns being transformed
    // stopping rules that read the error (REL / ABS): the error values come
    // back into page-locked slots, one per iteration, each marked by an event
    float *h_err = nullptr;
    cudaEvent_t ev_rb[2] = {nullptr, nullptr};
    int spec = -1;                 // iteration whose forward half is queued ahead of its decision
    long long slab_elems = 0;      // complex elements of each column buffer (0: a whole job)
    bool slab_copies = false;      // the z pass works on gathered copies (T allocated)
    float2 *T = nullptr;
};

namespace dwcu {

static int trace_cap(const dwcu_opts &s) { return std::max(1, std::max(s.n_iter, s.maxiter)); }

// ---- pass launchers

static int launch_lines(dwcu_job *j, const LinesPlan *p, const float2 *tw, long long n, long long line_stride,
                        long long outer_stride, long long nouter, long long ncols, int mode, float2 *data,
                        const char *axis, long long nin = -1, long long nout = -1, float2 *const *planes = nullptr,
                        long long col0 = 0)
{
    if (nin < 0) nin = n;
    if (nout < 0) nout = n;
    if (!p) return DWCU_SUCCESS;  // length-1 axis: identity
    LinesArgs a;
    a.data = data;
    a.otf = j->K;
    a.tw = tw;
    a.line_stride = line_stride;
    a.outer_stride = outer_stride;
    a.ncols = (int) ncols;
    a.ntiles = (int) ((ncols + p->T - 1) / p->T);
    a.mode = mode;
    a.nin = (int) nin;
    a.nout = (int) nout;
    a.planes = planes;
    a.col0 = col0;
    long long nb = (long long) a.ntiles * nouter;
    if (nb > 0x7fffffffLL) return fail(DWCU_ERROR_UNSUPPORTED, "grid too large");
    static const char *names[] = {"lines_fwd", "lines_inv", "lines_conv", "lines_conv_conj"};
    char nm[40];
    snprintf(nm, sizeof nm, "%s_%s", names[mode], axis);
    // algorithmic bytes: the elements read, the OTF (convolve modes), the elements written
    const double lines = (double) ncols * (double) nouter;
    const double bytes = 8.0 * lines * ((double) nin + (double) nout + (mode >= LINES_CONV ? (double) n : 0.0));
    ProfScope ps(nm, bytes, j->stream);
    p->launch(a, (int) nb, j->stream);
    CHECK_LAUNCH();
    return DWCU_SUCCESS;
}

// y transforms of the planes z < planes (default: all)
static int pass_y(dwcu_job *j, int mode, float2 *data, long long planes = -1)
{
    const Geometry &g = j->g;
    if (g.Y == 1) return DWCU_SUCCESS;
    if (planes < 0) planes = g.Z;
    if (g.ytp) {
        // one contiguous tile per (z, kx block): 4 lines of Y elements
        YArgs a;
        a.data = data;
        a.tw = j->tw_y;
        a.err = &j->sc->flags;
        a.ntiles = (int) (planes * g.NKB);
        a.dir = (mode == LINES_INV) ? +1 : -1;
        // the passes over the image planes only are timed as their own class
        const char *nm = mode == LINES_INV ? (planes < g.Z ? "y_inv_img" : "y_inv") : (planes < g.Z ? "y_fwd_img" : "y_fwd");
        ProfScope ps(nm, 16.0 * (double) g.NKB * KB * g.Y * planes, j->stream);
        g.ytp->launch(a, j->stream);
        CHECK_LAUNCH();
        return DWCU_SUCCESS;
    }
    // lines along y: 4 contiguous columns, stride KB, outer = (z, kx block)
    return launch_lines(j, g.yp, j->tw_y, g.Y, KB, g.Y * KB, planes * g.NKB, KB, mode, data, "y");
}
// z transforms; planes >= nin are taken as zero and not read, only planes
// < nout are written (defaults: all)
static int pass_z(dwcu_job *j, int mode, float2 *data, long long nin = -1, long long nout = -1)
{
    const Geometry &g = j->g;
    // lines along z: every (kx block, y, kx) of a plane is a column; stride = plane
    const long long plane = g.NKB * g.Y * KB;
    return launch_lines(j, g.zp, j->tw_z, g.Z, plane, 0, 1, plane, mode, data, "z", nin, nout);
}

static int pass_x(dwcu_job *j, int op, int r2c, float2 *S, const float *src, const float *srcp, float *dst,
                  double alpha, double alpha_next, long long tiles = -1, bool field = true)
{
    const Geometry &g = j->g;
    XArgs a;
    a.S = S;
    a.tw = j->tw_x;
    a.twL = j->tw_l;
    a.g = j->gimg;
    a.src = src;
    a.srcp = srcp;
    a.Wt = j->W;
    a.dst = dst;
    a.partial = j->partial;
    a.sc = j->sc;
    a.err = &j->sc->flags;
    a.X = g.XP;
    a.GP = g.GP;
    a.nkb = (int) g.NKB;
    a.ntiles = (int) (tiles < 0 ? j->nxb : tiles);
    a.Y = (int) g.Y;
    a.Z = (int) g.Z;
    a.M = (int) g.M;
    a.N = (int) g.N;
    a.P = (int) g.P;
    a.op = op;
    a.r2c = r2c;
    a.metric = j->s.metric;
    a.positivity = j->s.positivity;
    a.rl_clamp = 1;
    a.alpha = alpha;
    a.alpha_next = alpha_next;
    // the OTF is the shifted PSF, not a periodic field: no margins (`field`
    // false: the transform of the OTF into another buffer)
    const bool wrap = field && S != j->K;
    a.wrapx = (wrap && g.wx) ? 1 : 0;
    a.wM = (int) g.wM;
    a.hx = (int) g.hx;
    // algorithmic traffic of this launch
    static const char *names[] = {"x_fwd_copy", "x_fwd_ones", "x_fwd_shbp", "x_ratio_shb", "x_ratio_rl",
                                  "x_error", "x_update_shb", "x_update_rl", "x_weights", "x_store"};
    const double C = 8.0 * (double) (g.X / 2 + 1) * (double) (g.Y * g.Z);
    const double R = 4.0 * (double) g.X * (double) (g.Y * g.Z);  // algorithmic: the X used columns
    const double G = 4.0 * (double) (g.M * g.N * g.P);
    static const double real_in[] = {1, 0, 2, 0, 0, 0, 3, 2, 0, 0};
    static const double real_out[] = {0, 0, 0, 0, 0, 0, 1, 1, 1, 1};
    double bytes = (op >= XOP_RATIO_SHB ? C : 0.0) + (r2c ? C : 0.0) + (real_in[op] + real_out[op]) * R;
    if (op == XOP_UPDATE_SHB && !j->W) bytes -= R;
    if (op == XOP_UPDATE_RL && !j->W) bytes -= R;
    if (op == XOP_RATIO_SHB || op == XOP_RATIO_RL || op == XOP_ERROR_ONLY) {
        // only tiles holding image rows read their spectrum rows; the
        // launched tiles write theirs
        const long long Rr = g.xp->R, ytiles = (g.Y + Rr - 1) / Rr;
        const double rows_img = (double) g.P * (double) std::min(g.Y, ((g.N + Rr - 1) / Rr) * Rr);
        const double rows = (double) g.Y * (double) g.Z;
        const double launched = (double) std::min(rows, (double) a.ntiles / (double) ytiles * (double) g.Y);
        bytes = C * rows_img / rows + (r2c ? C * launched / rows : 0.0) + G;
    }
    ProfScope ps(names[op], bytes, j->stream);
    g.xp->launch(a, j->stream);
    CHECK_LAUNCH();
    if (r2c && wrap && (g.wy || g.wz)) {
        // periodic y/z: margin rows of the new spectrum copy the rows they wrap to
        const long long segs = g.Z * g.NKB * g.Y;
        const int blocks = (int) std::min<long long>(148 * 16, (segs + 255) / 256);
        k_wrap_rows<<<blocks, 256, 0, j->stream>>>(S, (int) g.Y, (int) g.Z, (int) g.NKB, (int) g.wN, (int) g.hy,
                                                   g.wy ? 1 : 0, (int) g.wP, (int) g.hz, g.wz ? 1 : 0);
        CHECK_LAUNCH();
    }
    return DWCU_SUCCESS;
}

static int err_final(dwcu_job *j, int k, long long tiles)
{
    const Geometry &g = j->g;
    k_err_final<<<1, kRedThreads, 0, j->stream>>>(j->partial, (int) tiles, (double) (g.M * g.N * g.P), j->err + k);
    CHECK_LAUNCH();
    return DWCU_SUCCESS;
}

#define TRY(x)                          \
    do {                                \
        int rc_ = (x);                  \
        if (rc_ != DWCU_SUCCESS) return rc_; \
    } while (0)

// method_shb.c:328-330: alpha = clamp((k - 1)/(k + 2), 0, alphamax)
static double shb_alpha(int k, float alphamax)
{
    double a = ((float) k - 1.0) / ((float) k + 2.0);
    if (a < 0) a = 0;
    if (a > alphamax) a = alphamax;
    return a;
}

static int conv(dwcu_job *j, int conj)
{
    TRY(pass_y(j, LINES_FWD, j->S));
    TRY(pass_z(j, conj ? LINES_CONV_CONJ : LINES_CONV, j->S));
    TRY(pass_y(j, LINES_INV, j->S));
    return DWCU_SUCCESS;
}

// The iteration's convolutions, pruned to the planes that matter.  The
// forward one (y = K p) is only read on the image (z < P): its z pass writes
// planes z < P and its inverse y pass transforms only those.  The ratio that
// the back-projection transforms is zero outside the image for SHB
// (method_shb.c:44-46), so its planes z >= P are zero: the forward y pass
// skips them and the z pass reads them as zero.  (RL's ratio is 1e-6 there,
// so its back-projection stays complete.)
static int conv_forward(dwcu_job *j)
{
    const Geometry &g = j->g;
    TRY(pass_y(j, LINES_FWD, j->S));
    TRY(pass_z(j, LINES_CONV, j->S, g.Z, g.P));
    TRY(pass_y(j, LINES_INV, j->S, g.P));
    return DWCU_SUCCESS;
}
static int conv_backward(dwcu_job *j)
{
    const Geometry &g = j->g;
    // (a periodic z copies image planes into its margins: no zero planes)
    if (j->s.method != DWCU_METHOD_SHB || g.wz) return conv(j, 1);
    TRY(pass_y(j, LINES_FWD, j->S, g.P));
    TRY(pass_z(j, LINES_CONV_CONJ, j->S, g.P, g.Z));
    TRY(pass_y(j, LINES_INV, j->S));
    return DWCU_SUCCESS;
}

// forward half of iteration k: y = K p_k, error_k; when `ratio`, also the
// ratio's transform into S.  The x pass runs the tiles of planes z < P only
// when nothing reads the other planes (SHB, or the error alone).
static int iter_forward(dwcu_job *j, int k, bool ratio)
{
    const Geometry &g = j->g;
    const bool shb = (j->s.method == DWCU_METHOD_SHB);
    TRY(conv_forward(j));
    int op = ratio ? (shb ? XOP_RATIO_SHB : XOP_RATIO_RL) : XOP_ERROR_ONLY;
    const long long ytiles = (g.Y + g.xp->R - 1) / g.xp->R;
    // planes z >= P are read later by RL, and by a periodic z (its margins)
    const long long tiles = (op == XOP_RATIO_RL || g.wz) ? j->nxb : g.P * ytiles;
    TRY(pass_x(j, op, ratio ? 1 : 0, j->S, nullptr, nullptr, nullptr, 0, 0, tiles));
    TRY(err_final(j, k, tiles));
    return DWCU_SUCCESS;
}

// back-projection half of iteration k: x_{k+1}; with `next`, also the
// transform of the next iteration's input into S
static int iter_backward(dwcu_job *j, int k, bool next)
{
    const bool shb = (j->s.method == DWCU_METHOD_SHB);
    TRY(conv_backward(j));
    if (shb) {
        TRY(pass_x(j, XOP_UPDATE_SHB, next ? 1 : 0, j->S, j->xa, j->xb, j->xb, shb_alpha(k, j->s.alphamax),
                   shb_alpha(k + 1, j->s.alphamax)));
        std::swap(j->xa, j->xb);  // xa = x_{k+1}, xb = x_k
    } else {
        TRY(pass_x(j, XOP_UPDATE_RL, next ? 1 : 0, j->S, j->xa, nullptr, j->xa, 0, 0));
    }
    return DWCU_SUCCESS;
}

// transform of iteration k's input (p_k for SHB, x_k for RL) into S
static int iter_input(dwcu_job *j, int k)
{
    if (j->s.method == DWCU_METHOD_SHB)
        return pass_x(j, XOP_FWD_SHBP, 1, j->S, j->xa, j->xb, nullptr, shb_alpha(k, j->s.alphamax), 0);
    return pass_x(j, XOP_FWD_COPY, 1, j->S, j->xa, nullptr, nullptr, 0, 0);
}

// ------------------------------------------------------------ guard bands
//
// A debugging aid in place of a memory checker: with guards on, every region
// of a job's block is preceded (and the last one followed) by kGuardBytes of
// a fixed pattern, written when the job is created and compared when it is
// destroyed; a write past the end of a region, or before its start, shows up
// as a changed guard (counted, and reported on stderr).  Mode 2 also
// overwrites one byte of the first guard from the host after filling it, so
// that a test can see the check find a change.
static std::atomic<int> g_guard_mode{0};
static std::atomic<long long> g_guard_violations{0};
constexpr size_t kGuardBytes = 4096;
constexpr int kGuardByte = 0xA5;

static int alloc_job(dwcu_job *j)
{
    const Geometry &g = j->g;
    const int guard_mode = g_guard_mode.load();
    // the x pass stages R rows per tile; a partial last tile reads (and
    // never uses) one row past the end, so every staged array gets a spare row
    const size_t R = sizeof(float) * (size_t) (g.real_elems() + g.XP);
    const size_t C = sizeof(float2) * (size_t) (g.spec_elems() + 8 * KB);
    const size_t G = sizeof(float) * (size_t) (g.GP * g.N * g.P + g.GP);
    j->nxb = x_blocks(g);
    j->n_spart = (int) std::min<long long>(1024, g.N * g.P);
    const long long npsf = g.pM * g.pN * g.pP;
    j->n_apart = (int) std::min<long long>(1024, (npsf + 4095) / 4096);
    const bool need_w = j->s.border_quality > 0;
    size_t off = 0;
    j->guards.clear();
    auto take = [&](size_t b) {
        if (guard_mode) {
            j->guards.push_back(off);
            off += kGuardBytes;
        }
        size_t o = off;
        off += align256(b);
        return o;
    };
    const size_t CK = j->slab_elems ? sizeof(float2) * (size_t) j->slab_elems : C;
    size_t o_g = take(G), o_S = take(C), o_K = take(CK), o_xa = take(R), o_xb = take(R);
    size_t o_T = (j->slab_elems && j->slab_copies) ? take(CK) : 0;
    size_t o_W = need_w ? take(R) : 0;
    size_t o_part = take(sizeof(double) * (size_t) j->nxb);
    size_t o_sc = take(sizeof(JobScalars));
    size_t o_err = take(sizeof(float) * (size_t) trace_cap(j->s));
    size_t o_amax = take(sizeof(long long));
    size_t o_sp = take(sizeof(StatsPartial) * (size_t) j->n_spart);
    size_t o_ap = take(sizeof(ArgmaxPartial) * (size_t) j->n_apart);
    size_t o_psf = take(sizeof(float) * (size_t) npsf);
    if (guard_mode) {
        j->guards.push_back(off);
        off += kGuardBytes;
    }
    j->bytes = off;
    j->block = block_get(j->s.device, off);
    if (!j->block)
        return fail(DWCU_ERROR_OUT_OF_MEMORY, "cudaMalloc of %.3f GB for the job failed", off / 1e9);
    j->base = j->block->ptr;
    char *b = j->base;
    j->gimg = (float *) (b + o_g);
    j->S = (float2 *) (b + o_S);
    j->K = (float2 *) (b + o_K);
    j->T = (j->slab_elems && j->slab_copies) ? (float2 *) (b + o_T) : nullptr;
    j->xa = (float *) (b + o_xa);
    j->xb = (float *) (b + o_xb);
    j->W = need_w ? (float *) (b + o_W) : nullptr;
    j->partial = (double *) (b + o_part);
    j->sc = (JobScalars *) (b + o_sc);
    j->err = (float *) (b + o_err);
    j->amax = (long long *) (b + o_amax);
    j->spart = (StatsPartial *) (b + o_sp);
    j->apart = (ArgmaxPartial *) (b + o_ap);
    j->psf_dev = (float *) (b + o_psf);
    for (size_t go : j->guards)
        if (cudaMemsetAsync(b + go, kGuardByte, kGuardBytes, j->stream) != cudaSuccess)
            return fail(DWCU_ERROR_CUDA, "filling a guard band failed");
    if (guard_mode == 2 && !j->guards.empty() && cudaMemsetAsync(b + j->guards[0], 0, 1, j->stream) != cudaSuccess)
        return fail(DWCU_ERROR_CUDA, "marking a guard band failed");
    return DWCU_SUCCESS;
}

// compares the job's guard bands with the pattern (after its work is done)
static void check_guards(dwcu_job *j)
{
    if (j->guards.empty() || !j->base) return;
    std::vector<unsigned char> h(kGuardBytes);
    for (size_t i = 0; i < j->guards.size(); ++i) {
        if (cudaMemcpy(h.data(), j->base + j->guards[i], kGuardBytes, cudaMemcpyDeviceToHost) != cudaSuccess) {
            cudaGetLastError();
            return;
        }
        size_t bad = 0;
        for (unsigned char c : h) bad += (c != (unsigned char) kGuardByte);
        if (bad) {
            ++g_guard_violations;
            fprintf(stderr, "dwcu: guard band %zu of a %lld x %lld x %lld job changed (%zu bytes)\n", i,
                    (long long) j->g.M, (long long) j->g.N, (long long) j->g.P, bad);
        }
    }
}

// ------------------------------------------------------------ autotuning
//
// tune_measure times the candidate plans of one transform length and pass
// kind (tune.cu keeps the choices).  Each candidate runs the pass it would
// run in an iteration on a synthetic volume of about kTuneElems complex
// elements: the z pass's convolve mode (lines), the persistent y pass in both
// directions (y), the SHB ratio and update x passes (x); one warm-up launch,
// then kTuneReps launches between CUDA events, on a stream of the tuner's
// own.  The volume is filled so that the ratio pass takes its usual branches
// (a positive image, a large constant term in every spectrum row, so that
// the blurred estimate is positive).  The scratch memory (a few hundred MB)
// is allocated for the measurement and freed after it.

static std::mutex g_tune_mu;
constexpr long long kTuneElems = 8LL << 20;  // complex elements of the synthetic spectrum (64 MB)
constexpr int kTuneReps = 4;

__device__ __forceinline__ unsigned tune_hash(unsigned long long i, unsigned seed)
{
    unsigned h = (unsigned) i * 2654435761u ^ (unsigned) (i >> 32) ^ seed;
    h ^= h >> 15;
    h *= 2246822519u;
    h ^= h >> 13;
    return h;
}

__global__ void k_tune_fill_real(float *p, long long n, float base, float amp, unsigned seed)
{
    for (long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x; i < n; i += (long long) gridDim.x * blockDim.x)
        p[i] = base + amp * (float) (tune_hash((unsigned long long) i, seed) & 0xffffu) * (1.f / 65536.f);
}

// blocked spectrum: a large real term at kx = 0 of every row, small noise elsewhere
__global__ void k_tune_fill_spec(float2 *S, long long n, int Y, int nkb, float dc, unsigned seed)
{
    for (long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x; i < n; i += (long long) gridDim.x * blockDim.x) {
        const int ki = (int) (i % KB);
        const int kb = (int) ((i / KB / Y) % nkb);
        const unsigned h = tune_hash((unsigned long long) i, seed);
        S[i] = (kb == 0 && ki == 0) ? make_float2(dc, 0.f)
                                    : make_float2((float) (h & 0xffffu) * (1.f / 65536.f) - 0.5f,
                                                  (float) (h >> 16) * (1.f / 65536.f) - 0.5f);
    }
}

static int tune_measure(DeviceCtx *ctx, int kind, int n, std::vector<float> &ms)
{
    const int cnt = (int) ms.size();
    std::fill(ms.begin(), ms.end(), -1.f);
    // a synthetic job of the pass's length, without OTF or weights set-up
    dwcu_job jj{};
    dwcu_opts_init(&jj.s);
    jj.s.device = ctx->device;
    jj.ctx = ctx;
    Geometry &g = jj.g;
    size_t spec = 0, real = 0, gbytes = 0;
    long long rows = 0;
    if (kind == DWCU_PLAN_LINES) {
        // z lines of length n over planes of 128 complex columns x Y rows
        g.X = 254; g.NKB = 32; g.Z = n;
        g.Y = std::max<long long>(1, kTuneElems / (n * g.NKB * KB));
        spec = sizeof(float2) * (size_t) (g.spec_elems() + 8 * KB);
    } else if (kind == DWCU_PLAN_Y) {
        g.X = 254; g.NKB = 32; g.Y = n;
        g.Z = std::max<long long>(1, kTuneElems / (n * g.NKB * KB));
        spec = sizeof(float2) * (size_t) (g.spec_elems() + 8 * KB);
    } else {
        // x rows of length 2n, every row and column inside the image
        const XPlan *p0 = x_plan(n, 0);
        if (!p0) return fail(DWCU_ERROR_UNSUPPORTED, "no x plan of length %d", n);
        g.X = 2LL * n; g.XP = (g.X + 3) & ~3LL; g.GP = g.XP;
        g.NKB = (n + 1 + KB - 1) / KB;
        rows = std::max<long long>(p0->R, kTuneElems / (g.NKB * KB));
        rows = (rows + p0->R - 1) / p0->R * p0->R;
        g.Y = rows; g.Z = 1;
        g.M = g.X; g.N = g.Y; g.P = 1;
        g.xp = p0;
        spec = sizeof(float2) * (size_t) (g.spec_elems() + 8 * KB);
        real = sizeof(float) * (size_t) (g.real_elems() + g.XP);
        gbytes = real;
    }
    g.wM = g.X; g.wN = g.Y; g.wP = g.Z;
    const long long nxb = kind == DWCU_PLAN_X ? x_blocks(g) : 0;
    size_t off = 0;
    auto take = [&](size_t b) { size_t o = off; off += align256(b); return o; };
    const size_t o_S = take(spec), o_K = kind == DWCU_PLAN_LINES ? take(spec) : 0;
    const size_t o_g = take(gbytes), o_xa = take(real), o_xb = take(real), o_W = take(real), o_xd = take(real);
    const size_t o_part = take(sizeof(double) * (size_t) (nxb + 1));
    const size_t o_sc = take(sizeof(JobScalars));
    char *base = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = DWCU_SUCCESS;
    if (cudaMalloc(&base, off) != cudaSuccess) {
        cudaGetLastError();
        return fail(DWCU_ERROR_OUT_OF_MEMORY, "no device memory for the tuning volume");
    }
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
        cudaEventCreate(&e1) != cudaSuccess)
        rc = fail(DWCU_ERROR_CUDA, "tuning stream or events could not be created");
    jj.stream = st;
    jj.S = (float2 *) (base + o_S);
    jj.K = kind == DWCU_PLAN_LINES ? (float2 *) (base + o_K) : nullptr;
    jj.sc = (JobScalars *) (base + o_sc);
    if (kind == DWCU_PLAN_X) {
        jj.gimg = (float *) (base + o_g);
        jj.xa = (float *) (base + o_xa);
        jj.xb = (float *) (base + o_xb);
        jj.W = (float *) (base + o_W);
        jj.partial = (double *) (base + o_part);
        jj.nxb = nxb;
    }
    if (rc == DWCU_SUCCESS) rc = get_twiddles(ctx, kind == DWCU_PLAN_X ? g.X : n, kind == DWCU_PLAN_X ? &jj.tw_x : kind == DWCU_PLAN_Y ? &jj.tw_y : &jj.tw_z);
    if (rc == DWCU_SUCCESS && kind == DWCU_PLAN_X) rc = get_twiddles(ctx, n, &jj.tw_l);
    if (rc == DWCU_SUCCESS) {
        const long long ns = g.spec_elems();
        k_tune_fill_spec<<<592, 256, 0, st>>>(jj.S, ns, (int) g.Y, (int) g.NKB, 50.f * (float) g.X, 1u);
        if (jj.K) k_tune_fill_spec<<<592, 256, 0, st>>>(jj.K, ns, (int) g.Y, (int) g.NKB, 1.f, 2u);
        if (kind == DWCU_PLAN_X) {
            const long long nr = g.real_elems();
            k_tune_fill_real<<<592, 256, 0, st>>>(jj.gimg, nr, 50.f, 100.f, 3u);
            k_tune_fill_real<<<592, 256, 0, st>>>(jj.xa, nr, 20.f, 10.f, 4u);
            k_tune_fill_real<<<592, 256, 0, st>>>(jj.xb, nr, 20.f, 10.f, 5u);
            k_tune_fill_real<<<592, 256, 0, st>>>(jj.W, nr, 0.5f, 1.f, 6u);
        }
        if (cudaMemsetAsync(jj.sc, 0, sizeof(JobScalars), st) != cudaSuccess || cudaGetLastError() != cudaSuccess)
            rc = fail(DWCU_ERROR_CUDA, "filling the tuning volume failed");
    }
    g_tuning = true;
    auto run_pass = [&]() -> int {
        if (kind == DWCU_PLAN_LINES) return pass_z(&jj, LINES_CONV, jj.S);
        if (kind == DWCU_PLAN_Y) {
            TRY(pass_y(&jj, LINES_FWD, jj.S));
            return pass_y(&jj, LINES_INV, jj.S);
        }
        TRY(pass_x(&jj, XOP_RATIO_SHB, 1, jj.S, nullptr, nullptr, nullptr, 0, 0, jj.nxb));
        return pass_x(&jj, XOP_UPDATE_SHB, 1, jj.S, jj.xa, jj.xb, (float *) (base + o_xd), 0.5, 0.6);
    };
    for (int c = 0; c < cnt && rc == DWCU_SUCCESS; ++c) {
        if (kind == DWCU_PLAN_LINES) g.zp = lines_plan(n, c);
        else if (kind == DWCU_PLAN_Y) g.ytp = y_plan(n, c);
        else g.xp = x_plan(n, c);
        if ((kind == DWCU_PLAN_LINES && !g.zp) || (kind == DWCU_PLAN_Y && !g.ytp) || (kind == DWCU_PLAN_X && !g.xp)) {
            rc = fail(DWCU_ERROR_INTERNAL, "missing tuning candidate %d of length %d", c, n);
            break;
        }
        rc = run_pass();  // warm-up (also sets the kernel's shared-memory attribute)
        if (rc == DWCU_SUCCESS && cudaEventRecord(e0, st) != cudaSuccess) rc = fail(DWCU_ERROR_CUDA, "event record failed");
        for (int r = 0; r < kTuneReps && rc == DWCU_SUCCESS; ++r) rc = run_pass();
        if (rc == DWCU_SUCCESS && cudaEventRecord(e1, st) != cudaSuccess) rc = fail(DWCU_ERROR_CUDA, "event record failed");
        float t = 0.f;
        if (rc == DWCU_SUCCESS && (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&t, e0, e1) != cudaSuccess))
            rc = fail(DWCU_ERROR_CUDA, "timing a tuning candidate failed");
        if (rc == DWCU_SUCCESS) ms[(size_t) c] = t / (float) kTuneReps;
    }
    g_tuning = false;
    // a bounded wait that gave up makes the measurement worthless
    JobScalars hs{};
    if (st) cudaStreamSynchronize(st);
    if (rc == DWCU_SUCCESS && cudaMemcpy(&hs, jj.sc, sizeof hs, cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = fail(DWCU_ERROR_CUDA, "reading the tuning flags failed");
    if (rc == DWCU_SUCCESS && (hs.flags & ~0xff))
        rc = fail(DWCU_ERROR_TIMEOUT, "a bounded wait gave up while tuning length %d", n);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
    cudaFree(base);
    return rc;
}

// the recorded choice of (device, kind, n), measured now if there is none
// and tuning is on; 0 (the heuristic plan) when the measurement fails
static int tuned_choice(DeviceCtx *ctx, int kind, int n, int *rc_out = nullptr)
{
    const int cnt = tune_plan_count(kind, n);
    if (cnt <= 1) return 0;
    int c = tune_lookup(ctx->device, kind, n);
    if (c >= 0 && c < cnt) return c;
    if (tune_mode() == DWCU_TUNE_OFF && !rc_out) return 0;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    c = tune_lookup(ctx->device, kind, n);  // measured meanwhile by another thread
    if (c >= 0 && c < cnt) return c;
    std::vector<float> ms((size_t) cnt, -1.f);
    const std::string saved = g_last_error;
    const int rc = tune_measure(ctx, kind, n, ms);
    if (rc_out) *rc_out = rc;
    if (rc != DWCU_SUCCESS) {
        cudaGetLastError();
        if (!rc_out) g_last_error = saved;
        return 0;
    }
    c = tune_select_idx(ms.data(), cnt, tune_margin());
    tune_record(ctx->device, kind, n, ms, c);
    return c;
}

// the geometry's plans: candidate 0 from make_geometry, replaced by the
// tuned choice of each pass's length (measure: false -- recorded choices
// only, e.g. an imported plan table, never a new measurement)
static void tune_geometry(DeviceCtx *ctx, Geometry &g, bool measure = true)
{
    auto choice = [&](int kind, int n) {
        if (measure) return tuned_choice(ctx, kind, n);
        const int c = tune_lookup(ctx->device, kind, n);
        return c >= 0 && c < tune_plan_count(kind, n) ? c : 0;
    };
    const int nx = (int) (g.X / 2);
    if (const XPlan *p = x_plan(nx, choice(DWCU_PLAN_X, nx))) g.xp = p;
    if (g.ytp) {
        if (const YPlan *p = y_plan((int) g.Y, choice(DWCU_PLAN_Y, (int) g.Y))) g.ytp = p;
    } else if (g.yp) {
        if (const LinesPlan *p = lines_plan((int) g.Y, choice(DWCU_PLAN_LINES, (int) g.Y))) g.yp = p;
    }
    if (const LinesPlan *p = lines_plan((int) g.Z, choice(DWCU_PLAN_LINES, (int) g.Z))) g.zp = p;
}

static long long job_bytes_estimate(const Geometry &g, const dwcu_opts &s)
{
    const long long R = 4LL * g.real_elems();
    const long long C = 8LL * g.spec_elems();
    const long long G = 4LL * g.GP * g.N * g.P;
    return G + 2 * C + (s.border_quality > 0 ? 3 : 2) * R + 8LL * ((g.Y * g.Z) / 2 + 1) +
           4LL * g.pM * g.pN * g.pP + (1 << 20);
}

static int check_opts(const dwcu_opts &s)
{
    if (s.method != DWCU_METHOD_SHB && s.method != DWCU_METHOD_RL)
        return fail(DWCU_ERROR_INVALID_VALUE, "method must be SHB (2) or RL (0), got %d", s.method);
    if (s.iter_type < 0 || s.iter_type > 2) return fail(DWCU_ERROR_INVALID_VALUE, "bad iter_type %d", s.iter_type);
    if (s.n_iter < 0 || s.maxiter < 0) return fail(DWCU_ERROR_INVALID_VALUE, "negative iteration count");
    if (s.start_condition != DWCU_START_FLAT && s.start_condition != DWCU_START_IDENTITY &&
        s.start_condition != DWCU_START_LP)
        return fail(DWCU_ERROR_INVALID_VALUE, "bad start_condition %d", s.start_condition);
    if (s.metric != DWCU_METRIC_IDIV && s.metric != DWCU_METRIC_MSE)
        return fail(DWCU_ERROR_INVALID_VALUE, "bad metric %d", s.metric);
    return DWCU_SUCCESS;
}

static int job_create(long long M, long long N, long long P, long long pM, long long pN, long long pP,
                      const dwcu_opts *s, dwcu_job **out)
{
    *out = nullptr;
    if (!s) return fail(DWCU_ERROR_INVALID_VALUE, "opts is NULL");
    TRY(check_opts(*s));
    Geometry g;
    TRY(make_geometry(M, N, P, pM, pN, pP, s->border_quality, g));
    DeviceCtx *ctx = nullptr;
    TRY(get_ctx(s->device, &ctx));
    CU(cudaSetDevice(s->device));
    tune_geometry(ctx, g);
    dwcu_job *j = new dwcu_job();
    j->s = *s;
    j->g = g;
    j->ctx = ctx;
    j->stream = ctx->stream;
    int rc = alloc_job(j);
    if (rc == DWCU_SUCCESS) rc = get_twiddles(ctx, g.X, &j->tw_x);
    if (rc == DWCU_SUCCESS) rc = get_twiddles(ctx, g.X / 2, &j->tw_l);
    if (rc == DWCU_SUCCESS && g.Y > 1) rc = get_twiddles(ctx, g.Y, &j->tw_y);
    if (rc == DWCU_SUCCESS) rc = get_twiddles(ctx, g.Z, &j->tw_z);
    if (rc == DWCU_SUCCESS &&
        (cudaEventCreate(&j->ev0) != cudaSuccess || cudaEventCreate(&j->ev1) != cudaSuccess ||
         cudaEventCreate(&j->ev2) != cudaSuccess))
        rc = fail(DWCU_ERROR_CUDA, "event creation failed");
    if (rc == DWCU_SUCCESS && s->iter_type != DWCU_ITER_FIXED &&
        (cudaMallocHost(&j->h_err, sizeof(float) * (size_t) trace_cap(*s)) != cudaSuccess ||
         cudaEventCreateWithFlags(&j->ev_rb[0], cudaEventDisableTiming) != cudaSuccess ||
         cudaEventCreateWithFlags(&j->ev_rb[1], cudaEventDisableTiming) != cudaSuccess))
        rc = fail(DWCU_ERROR_CUDA, "error read-back slots could not be set up");
    if (rc != DWCU_SUCCESS) {
        dwcu_job_destroy(j);
        return rc;
    }
    j->trace.assign((size_t) trace_cap(*s), 0.f);
    *out = j;
    return DWCU_SUCCESS;
}

// image (compact) into the job's pitched buffer, PSF into staging; then
// statistics, OTF, weights and the start estimate (method_shb.c:108-296)
static int job_setup(dwcu_job *j, const float *im, const float *psf, bool on_device)
{
    PhaseRange pr("dwcu job setup");
    const Geometry &g = j->g;
    CU(cudaSetDevice(j->s.device));
    cudaStream_t st = j->stream;
    CU(cudaEventRecord(j->ev0, st));
    const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    // From host memory the image crosses PCIe on the device's copy stream
    // while the OTF and the weights (which need only the image's size) are
    // computed; the statistics wait for it (ev2 marks it; the result
    // records ev2 again).  The PSF goes first: copies in one direction share
    // one copy engine, and the OTF needs the PSF.
    const long long npsf = g.pM * g.pN * g.pP;
    CU(cudaMemcpyAsync(j->psf_dev, psf, sizeof(float) * npsf, kind, st));
    CU(cudaMemsetAsync(j->sc, 0, sizeof(JobScalars), st));
    cudaStream_t cs = on_device ? st : j->ctx->copy;
    if (cs != st) CU(cudaStreamWaitEvent(cs, j->ev0, 0));
    CU(cudaMemcpy2DAsync(j->gimg, sizeof(float) * g.GP, im, sizeof(float) * g.M, sizeof(float) * g.M, g.N * g.P,
                         kind, cs));
    if (cs != st) CU(cudaEventRecord(j->ev2, cs));

    // OTF: PSF with its first maximum at the origin, scaled by 1/(X*Y*Z)
    const long long per = (npsf + j->n_apart - 1) / j->n_apart;
    const int nab = (int) ((npsf + per - 1) / per);
    k_argmax_partial<<<nab, kRedThreads, 0, st>>>(j->psf_dev, npsf, per, j->apart, &j->sc->flags);
    CHECK_LAUNCH();
    k_argmax_final<<<1, 32, 0, st>>>(j->apart, nab, j->amax);
    CHECK_LAUNCH();
    if (g.wx || g.wy || g.wz) {
        // the periodic margins assume the PSF maximum within h of both ends
        long long am = 0;
        CU(cudaMemcpyAsync(&am, j->amax, sizeof am, cudaMemcpyDeviceToHost, st));
        CU(cudaStreamSynchronize(st));
        const long long ax = am % g.pM, ay = (am / g.pM) % g.pN, az = am / (g.pM * g.pN);
        auto off = [](long long a, long long p) { return std::max(a, p - 1 - a); };
        if ((g.wx && off(ax, g.pM) > g.hx) || (g.wy && off(ay, g.pN) > g.hy) || (g.wz && off(az, g.pP) > g.hz))
            return fail(DWCU_ERROR_UNSUPPORTED,
                        "border_quality %d with a job size that has no exact transform needs the PSF maximum at "
                        "its centre (maximum at %lld, %lld, %lld of %lld x %lld x %lld)",
                        j->s.border_quality, ax, ay, az, g.pM, g.pN, g.pP);
    }
    const size_t R = sizeof(float) * (size_t) g.real_elems();
    CU(cudaMemsetAsync(j->S, 0, sizeof(float2) * (size_t) g.spec_elems(), st));
    CU(cudaMemsetAsync(j->K, 0, sizeof(float2) * (size_t) g.spec_elems(), st));
    CU(cudaMemsetAsync(j->xb, 0, R, st));
    const float scale = (float) (1.0 / ((double) g.X * (double) g.Y * (double) g.Z));
    k_psf_embed<<<(int) std::min<long long>(4096, (npsf + 255) / 256), 256, 0, st>>>(
        j->psf_dev, (int) g.pM, (int) g.pN, (int) g.pP, j->amax, j->xb, (int) g.X, (int) g.Y, (int) g.Z,
        (int) g.XP, scale);
    CHECK_LAUNCH();
    TRY(pass_x(j, XOP_FWD_COPY, 1, j->K, j->xb, nullptr, nullptr, 0, 0));
    TRY(pass_y(j, LINES_FWD, j->K));
    TRY(pass_z(j, LINES_FWD, j->K));

    // Bertero weights: W = 1/P1 where P1 = K^T 1_image > 0.01 (method_shb.c:216-235)
    if (j->W) {
        TRY(pass_x(j, XOP_FWD_ONES, 1, j->S, nullptr, nullptr, nullptr, 0, 0));
        TRY(conv(j, 1));
        TRY(pass_x(j, XOP_WEIGHTS, 0, j->S, nullptr, nullptr, j->W, 0, 0));
    }

    // background and start value (the image is on the device from here on)
    if (cs != st) CU(cudaStreamWaitEvent(st, j->ev2, 0));
    {
        const long long nrows = g.N * g.P;
        const long long rpb = (nrows + j->n_spart - 1) / j->n_spart;
        const int nsb = (int) ((nrows + rpb - 1) / rpb);
        k_stats_partial<<<nsb, kRedThreads, 0, st>>>(j->gimg, g.GP, (int) g.M, nrows, rpb, j->spart);
        CHECK_LAUNCH();
        k_stats_final<<<1, kRedThreads, 0, st>>>(j->spart, nsb, j->sc, j->s.bg_auto, j->s.bg,
                                                 (unsigned long long) (g.wM * g.wN * g.wP));
        CHECK_LAUNCH();
    }

    // start estimate (method_shb.c:264-276); x_{-1} = x_0
    const long long nv = g.real_elems();
    const int fb = (int) std::min<long long>(148 * 16, (nv + 255) / 256);
    if (j->s.start_condition == DWCU_START_FLAT) {
        k_fill_scalar<<<fb, 256, 0, st>>>(j->xa, nv, j->sc);
        CHECK_LAUNCH();
    } else if (j->s.start_condition == DWCU_START_LP) {
        // method_shb.c:278-285, method_rl.c:290-297: the image smoothed by
        // fim_gsmooth(sigma 8), inserted at the corner.  x_{k-1} and the
        // spectrum are free here and hold the intermediate volumes.
        const long long nimg = g.M * g.N * g.P;
        const int gb = (int) std::min<long long>(148 * 16, (nimg + 255) / 256);
        float *t1 = j->xb, *t2 = reinterpret_cast<float *>(j->S);
        GaussTaps K = gauss_taps(8.0f);
        CU(cudaMemcpy2DAsync(t2, sizeof(float) * g.M, j->gimg, sizeof(float) * g.GP, sizeof(float) * g.M,
                             g.N * g.P, cudaMemcpyDeviceToDevice, st));
        k_gsmooth_axis<<<gb, 256, 0, st>>>(t2, t1, (int) g.M, (int) g.N, (int) g.P, 0, K);
        CHECK_LAUNCH();
        k_gsmooth_axis<<<gb, 256, 0, st>>>(t1, t2, (int) g.M, (int) g.N, (int) g.P, 1, K);
        CHECK_LAUNCH();
        const float *lp = t2;
        if (g.P > 1) {
            // fim_gsmooth_aniso trims the z kernel to at most 2P-1 taps
            GaussTaps Kz = K;
            int off = 0;
            while (Kz.n > 2 * g.P - 1) {
                ++off;
                Kz.n -= 2;
            }
            for (int i = 0; i < Kz.n; ++i) Kz.k[i] = K.k[i + off];
            k_gsmooth_axis<<<gb, 256, 0, st>>>(t2, t1, (int) g.M, (int) g.N, (int) g.P, 2, Kz);
            CHECK_LAUNCH();
            lp = t1;
        }
        CU(cudaMemsetAsync(j->xa, 0, R, st));
        k_embed_image<<<fb, 256, 0, st>>>(lp, g.M, (int) g.M, (int) g.N, (int) g.P, j->xa, (int) g.XP, (int) g.Y);
        CHECK_LAUNCH();
    } else {
        CU(cudaMemsetAsync(j->xa, 0, R, st));
        k_embed_image<<<fb, 256, 0, st>>>(j->gimg, g.GP, (int) g.M, (int) g.N, (int) g.P, j->xa, (int) g.XP,
                                          (int) g.Y);
        CHECK_LAUNCH();
    }
    if (j->s.method == DWCU_METHOD_SHB) CU(cudaMemcpyAsync(j->xb, j->xa, R, cudaMemcpyDeviceToDevice, st));

    // input flags (non-finite values) are checked once, here
    JobScalars hs;
    CU(cudaMemcpyAsync(&hs, j->sc, sizeof hs, cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    if (hs.flags & 1) return fail(DWCU_ERROR_INPUT, "the image contains non-finite values");
    if (hs.flags & 2) return fail(DWCU_ERROR_INPUT, "the PSF contains non-finite values");
    if (j->s.bg_auto) j->s.bg = hs.bg;
    j->it.init(j->s);
    j->k_next = j->it.next();
    j->finished = (j->k_next < 0);
    j->spectrum_ready = false;
    j->done_iters = 0;
    j->setup_done = true;
    CU(cudaEventRecord(j->ev1, st));
    return DWCU_SUCCESS;
}

// Enqueue iterations.  FIXED: no host synchronisation (and, if requested, the
// whole remaining loop as one CUDA graph).  REL/ABS: each error is read back
// before deciding whether the next iteration runs (dw.c:237-270).
static int job_step_impl(dwcu_job *j, int nmax, int *remaining);
static int job_step(dwcu_job *j, int nmax, int *remaining)
{
    PhaseRange pr("dwcu job iterations");
    auto t0 = std::chrono::steady_clock::now();
    int rc = job_step_impl(j, nmax, remaining);
    j->enqueue_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return rc;
}

static int job_step_impl(dwcu_job *j, int nmax, int *remaining)
{
    if (!j->setup_done) return fail(DWCU_ERROR_INVALID_VALUE, "job_step before job_setup");
    CU(cudaSetDevice(j->s.device));
    const bool shb = (j->s.method == DWCU_METHOD_SHB);
    const bool fixed = (j->s.iter_type == DWCU_ITER_FIXED);
    int ran = 0;
    auto run_one_fixed = [&](int k) -> int {
        const bool last = (k == j->it.niter - 1);
        if (!j->spectrum_ready) TRY(iter_input(j, k));
        // SHB's last update is discarded (method_shb.c:385-395): only its error is needed
        TRY(iter_forward(j, k, !(last && shb)));
        if (!(last && shb)) TRY(iter_backward(j, k, !last));
        j->spectrum_ready = !last;
        return DWCU_SUCCESS;
    };
    while (!j->finished && ran < nmax) {
        const int k = j->k_next;
        if (fixed) {
            bool prof_now;
            {
                std::lock_guard<std::mutex> lk(g_prof_mu);
                prof_now = g_prof_on;
            }
            // with kernel timing on, launches stay eager: timing events inside
            // a graph make every replay expensive on the host
            const bool use_graph = j->s.use_graph && !prof_now && nmax >= (j->it.niter - k) && (j->it.niter - k) > 1;
            if (use_graph) {
                // The whole remaining loop as one graph.  A graph captured
                // earlier on this memory block for the same sizes, options
                // and starting state is launched again (its kernels carry
                // the same pointers and parameters).
                bool prof;
                {
                    std::lock_guard<std::mutex> lk(g_prof_mu);
                    prof = g_prof_on;
                }
                char key[512];
                const Geometry &gg = j->g;
                snprintf(key, sizeof key,
                         "%lld %lld %lld %lld %lld %lld %lld %lld %lld|%d %d %d %d %d %d %d %a|%d %d %d %p %p|%p %p %p %p",
                         gg.M, gg.N, gg.P, gg.pM, gg.pN, gg.pP, gg.X, gg.Y, gg.Z, j->s.method, j->it.niter,
                         j->s.maxiter, k, j->s.metric, j->s.positivity, j->s.border_quality, (double) j->s.alphamax,
                         (int) j->spectrum_ready, (int) (j->W != nullptr), (int) prof, (void *) j->xa, (void *) j->xb,
                         (const void *) gg.xp, (const void *) gg.yp, (const void *) gg.zp, (const void *) gg.ytp);
                const std::string skey(key);
                cudaGraphExec_t ex = nullptr;
                auto hit = j->block->graphs.find(skey);
                long long kernels = 0;
                if (hit != j->block->graphs.end()) {
                    ex = hit->second.exec;
                    // the buffer roles the loop leaves behind (SHB swaps after
                    // every update; the last iteration has none)
                    if (shb)
                        for (int kk = k; kk < j->it.niter - 1; ++kk) std::swap(j->xa, j->xb);
                    g_launches += hit->second.kernels;
                    if (prof) {
                        // this replay re-records the graph's timing events
                        std::lock_guard<std::mutex> lk(g_prof_mu);
                        for (auto &r : hit->second.recs) g_prof_recs.push_back(r);
                    }
                } else {
                    auto t0 = std::chrono::steady_clock::now();
                    cudaGraph_t gr = nullptr;
                    CU(cudaStreamBeginCapture(j->stream, cudaStreamCaptureModeThreadLocal));
                    int rc = DWCU_SUCCESS;
                    const long long l0 = g_launches;
                    size_t r0;
                    {
                        std::lock_guard<std::mutex> lk(g_prof_mu);
                        r0 = g_prof_recs.size();
                    }
                    for (int kk = k; kk < j->it.niter && rc == DWCU_SUCCESS; ++kk) rc = run_one_fixed(kk);
                    kernels = g_launches - l0;
                    std::vector<ProfRec> grecs;
                    {
                        std::lock_guard<std::mutex> lk(g_prof_mu);
                        if (g_prof_recs.size() > r0) grecs.assign(g_prof_recs.begin() + (long) r0, g_prof_recs.end());
                    }
                    cudaError_t ce = cudaStreamEndCapture(j->stream, &gr);
                    if (rc != DWCU_SUCCESS) {
                        if (gr) cudaGraphDestroy(gr);
                        return rc;
                    }
                    if (ce != cudaSuccess)
                        return fail(DWCU_ERROR_CUDA, "graph capture failed: %s", cudaGetErrorString(ce));
                    auto t1 = std::chrono::steady_clock::now();
                    ce = cudaGraphInstantiate(&ex, gr, 0);
                    cudaGraphDestroy(gr);
                    if (ce != cudaSuccess)
                        return fail(DWCU_ERROR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(ce));
                    auto t2 = std::chrono::steady_clock::now();
                    if (trace_on())
                        fprintf(stderr, "dwcu: captured %lld kernels in %.1f ms, instantiated in %.1f ms\n", kernels,
                                std::chrono::duration<double, std::milli>(t1 - t0).count(),
                                std::chrono::duration<double, std::milli>(t2 - t1).count());
                    Block::Graph gent;
                    gent.exec = ex;
                    gent.kernels = kernels;
                    gent.recs = grecs;
                    j->block->graphs[skey] = gent;
                }
                CU(cudaGraphLaunch(ex, j->stream));  // its kernels are counted at capture (or replayed above)
                ran += j->it.niter - k;
                j->done_iters = j->it.niter;
                j->it.iter = j->it.niter;
                j->k_next = -1;
                j->finished = true;
                break;
            }
            TRY(run_one_fixed(k));
            ran++;
            j->done_iters = k + 1;
            j->k_next = (k + 1 < j->it.niter) ? k + 1 : -1;
            j->it.iter = k;
            if (j->k_next < 0) j->finished = true;
            continue;
        }
        // REL / ABS (dw.c:237-270): error k decides whether iteration k+1
        // runs.  Iteration k+1 (the back-projection of k and the forward
        // half of k+1) is queued before the host waits for error k, so the
        // GPU does not idle while the host reads and decides.  When the rule
        // stops at k, the queued work is dropped: SHB's result x_k goes back
        // to xa by swapping the estimates back, and RL's result x_{k+1} is
        // the back-projection already computed.
        auto queue_read = [&](int kk) -> int {
            CU(cudaMemcpyAsync(j->h_err + kk, j->err + kk, sizeof(float), cudaMemcpyDeviceToHost, j->stream));
            CU(cudaEventRecord(j->ev_rb[kk & 1], j->stream));
            return DWCU_SUCCESS;
        };
        if (j->spec != k) {
            if (!j->spectrum_ready) TRY(iter_input(j, k));
            TRY(iter_forward(j, k, true));
            TRY(queue_read(k));
        }
        const bool ahead = (k + 1 < j->it.niter);
        j->spec = -1;
        if (ahead) {
            TRY(iter_backward(j, k, true));
            TRY(iter_forward(j, k + 1, true));
            TRY(queue_read(k + 1));
            j->spec = k + 1;
        }
        CU(cudaEventSynchronize(j->ev_rb[k & 1]));
        const float e = j->h_err[k];
        j->it.set(e);
        j->trace[(size_t) k] = e;
        j->done_iters = k + 1;
        if (j->s.verbosity > 0) printf("Iteration %3d/%3d, %s=%.3e\n", k + 1, j->it.niter,
                                       j->s.metric == DWCU_METRIC_IDIV ? "Idiv" : "fMSE", e);
        const int kn = j->it.next();
        ran++;
        if (kn >= 0) {
            // kn == k + 1 (dw_iterator_next counts up), queued above
            j->spectrum_ready = false;
            j->k_next = kn;
        } else {
            if (ahead) {
                if (shb) std::swap(j->xa, j->xb);  // x_k back in xa
            } else if (!shb) {
                TRY(iter_backward(j, k, false));  // RL returns x_{k+1}
            }
            j->spec = -1;
            j->spectrum_ready = false;
            j->k_next = -1;
            j->finished = true;
        }
    }
    if (remaining) {
        if (j->finished) *remaining = 0;
        else *remaining = fixed ? (j->it.niter - j->k_next) : (j->it.niter - j->k_next);
    }
    return DWCU_SUCCESS;
}

// result: SHB's output is x_{N-1}, i.e. the estimate the last forward half
// read; RL's is x_N.  Both live in xa when the loop has finished.
static int job_result(dwcu_job *j, float *out, bool on_device, dwcu_opts *so)
{
    PhaseRange pr("dwcu job result");
    const Geometry &g = j->g;
    CU(cudaSetDevice(j->s.device));
    if (!j->finished) return fail(DWCU_ERROR_NOT_READY, "the job has iterations left");
    cudaStream_t st = j->stream;
    float *dout = out;
    float *tmp = nullptr;
    if (!on_device) {
        // crop on the device into the S buffer (free now), then one copy
        tmp = reinterpret_cast<float *>(j->S);
        dout = tmp;
    }
    const long long n = g.M * g.N * g.P;
    const int fb = (int) std::min<long long>(148 * 16, (n + 255) / 256);
    k_crop<<<fb, 256, 0, st>>>(j->xa, (int) g.XP, (int) g.Y, (int) g.M, (int) g.N, (int) g.P, dout);
    CHECK_LAUNCH();
    CU(cudaEventRecord(j->ev2, st));
    if (!on_device) CU(cudaMemcpyAsync(out, tmp, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
    const int nerr = j->done_iters;
    std::vector<float> errs((size_t) std::max(1, nerr));
    if (nerr > 0) CU(cudaMemcpyAsync(errs.data(), j->err, sizeof(float) * nerr, cudaMemcpyDeviceToHost, st));
    JobScalars hs{};
    CU(cudaMemcpyAsync(&hs, j->sc, sizeof hs, cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    if (hs.flags & ~3) return fail(DWCU_ERROR_TIMEOUT, "a bounded wait in a pass gave up (flags 0x%x)", hs.flags);
    if (so) {
        so->iterations_done = nerr;
        so->bg = j->s.bg;
        so->work[0] = g.X; so->work[1] = g.Y; so->work[2] = g.Z;
        float ms_setup = 0, ms_loop = 0;
        cudaEventElapsedTime(&ms_setup, j->ev0, j->ev1);
        cudaEventElapsedTime(&ms_loop, j->ev1, j->ev2);
        so->seconds_setup = ms_setup * 1e-3;
        so->seconds_iterate = ms_loop * 1e-3;
        so->seconds_enqueue = j->enqueue_s;
        if (so->error_trace)
            for (int i = 0; i < nerr && i < so->trace_capacity; ++i) so->error_trace[i] = errs[(size_t) i];
        if (j->s.verbosity > 0 && j->s.iter_type == DWCU_ITER_FIXED)
            for (int i = 0; i < nerr; ++i)
                printf("Iteration %3d/%3d, %s=%.3e\n", i + 1, nerr,
                       j->s.metric == DWCU_METRIC_IDIV ? "Idiv" : "fMSE", errs[(size_t) i]);
    }
    return DWCU_SUCCESS;
}

// Run a batch of set-up jobs to completion together.  Jobs with a fixed
// iteration count are captured into one CUDA graph with one stream per job:
// the graph holds independent chains, so small jobs (tiles, channels) share
// the GPU instead of running one after another.  Jobs with a REL/ABS stopping
// rule are stepped round-robin, one iteration each, on their own streams.
// padded job voxels from which one job's passes fill every SM
constexpr double kBatchLargeJob = 32.0 * 1024 * 1024;

static int batch_run(dwcu_job **jobs, int n, cudaStream_t origin)
{
    if (n <= 0) return DWCU_SUCCESS;
    const int dev = jobs[0]->s.device;
    for (int i = 0; i < n; ++i) {
        if (!jobs[i] || !jobs[i]->setup_done) return fail(DWCU_ERROR_INVALID_VALUE, "batch: job %d not set up", i);
        if (jobs[i]->s.device != dev) return fail(DWCU_ERROR_INVALID_VALUE, "batch: jobs on different devices");
    }
    CU(cudaSetDevice(dev));
    DeviceCtx *ctx = jobs[0]->ctx;
    if (!origin) origin = ctx->stream;
    // one stream per job (kept by the caller's jobs for the duration)
    std::vector<cudaStream_t> streams((size_t) n);
    std::vector<cudaStream_t> saved((size_t) n);
    for (int i = 0; i < n; ++i) {
        CU(cudaStreamCreateWithFlags(&streams[(size_t) i], cudaStreamNonBlocking));
        saved[(size_t) i] = jobs[i]->stream;
        jobs[i]->stream = streams[(size_t) i];
    }
    int rc = DWCU_SUCCESS;
    std::vector<int> fixed_idx, rel_idx;
    for (int i = 0; i < n; ++i) {
        if (jobs[i]->finished) continue;
        (jobs[i]->s.iter_type == DWCU_ITER_FIXED ? fixed_idx : rel_idx).push_back(i);
    }
    // prior work of every job (its setup) must finish before its chain runs
    cudaEvent_t fork = nullptr, done = nullptr;
    CU(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    CU(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
    for (int i = 0; i < n; ++i) {
        cudaEvent_t e = nullptr;
        cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
        cudaEventRecord(e, saved[(size_t) i]);
        cudaStreamWaitEvent(origin, e, 0);
        cudaEventDestroy(e);
    }
    if (!fixed_idx.empty()) {
        // Each job's remaining loop is one CUDA graph, cached on its memory
        // block (captured the first time a job of these sizes and options
        // runs on that block, replayed after that), launched on the job's own
        // stream, so small jobs run side by side.  Jobs that fill the GPU on
        // their own run one after another on one stream: side by side they
        // would only compete for the SMs and evict each other's data from L2
        // between passes.
        cudaEventRecord(fork, origin);
        int big_chain = -1;
        for (int i : fixed_idx) {
            dwcu_job *j = jobs[i];
            const double vox = (double) j->g.X * (double) j->g.Y * (double) j->g.Z;
            if (vox >= kBatchLargeJob) {
                if (big_chain < 0)
                    big_chain = i;
                else
                    j->stream = streams[(size_t) big_chain];
            }
            cudaStreamWaitEvent(j->stream, fork, 0);
            if (rc == DWCU_SUCCESS) rc = job_step_impl(j, 1 << 30, nullptr);
            cudaEventRecord(done, j->stream);
            cudaStreamWaitEvent(origin, done, 0);
        }
    }
    // stopping rules that read the error back: round-robin, one iteration at a time
    bool any = true;
    while (rc == DWCU_SUCCESS && any) {
        any = false;
        for (int i : rel_idx) {
            dwcu_job *j = jobs[i];
            if (j->finished) continue;
            if (rc == DWCU_SUCCESS) rc = job_step_impl(j, 1, nullptr);
            any = any || !j->finished;
        }
    }
    for (int i = 0; i < n; ++i) {
        cudaStreamSynchronize(streams[(size_t) i]);
        jobs[i]->stream = saved[(size_t) i];
        cudaStreamDestroy(streams[(size_t) i]);
    }
    cudaStreamSynchronize(origin);
    cudaEventDestroy(fork);
    cudaEventDestroy(done);
    return rc;
}

static int one_call(const float *im, long long M, long long N, long long P, const float *psf, long long pM,
                    long long pN, long long pP, dwcu_opts *s, float *out, bool on_device, cudaStream_t stream)
{
    if (!s || !im || !psf || !out) return fail(DWCU_ERROR_INVALID_VALUE, "NULL argument");
    s->iterations_done = 0;
    if (s->n_iter == 0) {
        // method_shb.c:101-105: nIter == 0 returns a copy of the image
        if (on_device) {
            CU(cudaSetDevice(s->device));
            CU(cudaMemcpyAsync(out, im, sizeof(float) * M * N * P, cudaMemcpyDeviceToDevice, stream));
            CU(cudaStreamSynchronize(stream));
        } else {
            memcpy(out, im, sizeof(float) * (size_t) (M * N * P));
        }
        return DWCU_SUCCESS;
    }
    dwcu_job *j = nullptr;
    TRY(job_create(M, N, P, pM, pN, pP, s, &j));
    if (on_device && stream) j->stream = stream;
    int rc = job_setup(j, im, psf, on_device);
    // a pageable result buffer is faulted in by a host thread while the
    // device iterates, so that the result copy does not wait for it
    std::thread prefault;
    if (!on_device) {
        cudaPointerAttributes pa;
        const bool locked = cudaPointerGetAttributes(&pa, out) == cudaSuccess && pa.type == cudaMemoryTypeHost;
        cudaGetLastError();
        const size_t n = (size_t) (M * N * P);
        const uintptr_t o0 = (uintptr_t) out, i0 = (uintptr_t) im, nb = sizeof(float) * n;
        const bool overlap = o0 < i0 + nb && i0 < o0 + nb;  // an in-place call
        if (!locked && !overlap && rc == DWCU_SUCCESS)
            prefault = std::thread([out, n]() {
                const size_t chunk = (size_t) 1 << 22;
                for (size_t i = 0; i < n; i += chunk) memset(out + i, 0, sizeof(float) * std::min(chunk, n - i));
            });
    }
    if (rc == DWCU_SUCCESS) rc = job_step(j, 1 << 30, nullptr);
    if (prefault.joinable()) prefault.join();
    if (rc == DWCU_SUCCESS) rc = job_result(j, out, on_device, s);
    if (rc == DWCU_SUCCESS && s->bg_auto) s->bg = j->s.bg;
    dwcu_job_destroy(j);
    return rc;
}

// standalone 3-D transforms on exact sizes (fft.c's fft()/ifft())
static int fft3d(const float *d_in, long long M, long long N, long long P, float *d_out, int device,
                 cudaStream_t stream, bool forward)
{
    if (!d_in || !d_out) return fail(DWCU_ERROR_INVALID_VALUE, "NULL argument");
    if (M < 2 || N < 1 || P < 1 || (M % 2)) return fail(DWCU_ERROR_INVALID_VALUE, "M must be even and >= 2");
    DeviceCtx *ctx = nullptr;
    TRY(get_ctx(device, &ctx));
    CU(cudaSetDevice(device));
    dwcu_job jj{};
    dwcu_job *j = &jj;
    dwcu_opts_init(&j->s);
    Geometry &g = j->g;
    g.M = M; g.N = N; g.P = P; g.pM = g.pN = g.pP = 1;
    g.wM = g.X = M; g.wN = g.Y = N; g.wP = g.Z = P;
    g.xp = find_x((int) (M / 2));
    g.yp = N > 1 ? find_lines((int) N) : nullptr;
    g.zp = find_lines((int) P);
    g.ytp = N > 1 ? find_y((int) N) : nullptr;
    if (!g.xp || (N > 1 && !g.yp) || !g.zp)
        return fail(DWCU_ERROR_UNSUPPORTED, "unsupported transform size %lld x %lld x %lld", M, N, P);
    g.XP = (M + 3) & ~3LL;
    g.NKB = (M / 2 + 1 + KB - 1) / KB;
    g.GP = (M + 3) & ~3LL;
    j->s.metric = DWCU_METRIC_IDIV;
    j->s.positivity = 1;
    j->ctx = ctx;
    j->stream = stream ? stream : ctx->stream;
    j->nxb = x_blocks(g);
    TRY(get_twiddles(ctx, g.X, &j->tw_x));
    TRY(get_twiddles(ctx, g.X / 2, &j->tw_l));
    if (N > 1) TRY(get_twiddles(ctx, N, &j->tw_y));
    TRY(get_twiddles(ctx, P, &j->tw_z));
    const size_t C = align256(sizeof(float2) * (size_t) (g.spec_elems() + 8 * KB));
    const size_t R = align256(sizeof(float) * (size_t) (g.real_elems() + g.XP));
    void *tmp = nullptr;
    CU(cudaMalloc(&tmp, C + R + 256));
    j->S = (float2 *) tmp;
    float *real = (float *) ((char *) tmp + C);
    j->sc = (JobScalars *) ((char *) tmp + C + R);
    j->K = nullptr;
    j->W = nullptr;
    j->partial = nullptr;
    int rc = DWCU_SUCCESS;
    const long long H = M / 2 + 1;
    const long long nspec = H * N * P;
    const int fb = (int) std::min<long long>(148 * 16, (nspec + 255) / 256);
    if (cudaMemsetAsync(tmp, 0, C + R + 256, j->stream) != cudaSuccess) rc = fail(DWCU_ERROR_CUDA, "memset");
    if (forward) {
        if (rc == DWCU_SUCCESS &&
            cudaMemcpy2DAsync(real, sizeof(float) * g.XP, d_in, sizeof(float) * M, sizeof(float) * M, N * P,
                              cudaMemcpyDeviceToDevice, j->stream) != cudaSuccess)
            rc = fail(DWCU_ERROR_CUDA, "copy failed");
        if (rc == DWCU_SUCCESS) rc = pass_x(j, XOP_FWD_COPY, 1, j->S, real, nullptr, nullptr, 0, 0);
        if (rc == DWCU_SUCCESS) rc = pass_y(j, LINES_FWD, j->S);
        if (rc == DWCU_SUCCESS) rc = pass_z(j, LINES_FWD, j->S);
        if (rc == DWCU_SUCCESS) {
            k_spec_unpack<<<fb, 256, 0, j->stream>>>(j->S, (int) H, (int) N, (int) P, (int) g.NKB,
                                                     reinterpret_cast<float2 *>(d_out));
            ++g_launches;
            if (cudaGetLastError() != cudaSuccess) rc = fail(DWCU_ERROR_CUDA, "unpack launch failed");
        }
    } else {
        k_spec_pack<<<fb, 256, 0, j->stream>>>(reinterpret_cast<const float2 *>(d_in), (int) H, (int) N, (int) P,
                                               (int) g.NKB, j->S);
        ++g_launches;
        if (cudaGetLastError() != cudaSuccess) rc = fail(DWCU_ERROR_CUDA, "pack launch failed");
        if (rc == DWCU_SUCCESS) rc = pass_z(j, LINES_INV, j->S);
        if (rc == DWCU_SUCCESS) rc = pass_y(j, LINES_INV, j->S);
        if (rc == DWCU_SUCCESS) rc = pass_x(j, XOP_STORE, 0, j->S, nullptr, nullptr, real, 0, 0);
        if (rc == DWCU_SUCCESS &&
            cudaMemcpy2DAsync(d_out, sizeof(float) * M, real, sizeof(float) * g.XP, sizeof(float) * M, N * P,
                              cudaMemcpyDeviceToDevice, j->stream) != cudaSuccess)
            rc = fail(DWCU_ERROR_CUDA, "copy failed");
    }
    cudaError_t e = cudaStreamSynchronize(j->stream);
    JobScalars hs{};
    if (e == cudaSuccess) e = cudaMemcpy(&hs, j->sc, sizeof hs, cudaMemcpyDeviceToHost);
    cudaFree(tmp);
    j->base = nullptr;
    j->ev0 = j->ev1 = j->ev2 = nullptr;
    j->stream = nullptr;
    if (rc != DWCU_SUCCESS) return rc;
    if (e != cudaSuccess) return fail(DWCU_ERROR_CUDA, "transform failed: %s", cudaGetErrorString(e));
    if (hs.flags & ~3) return fail(DWCU_ERROR_TIMEOUT, "a bounded wait in a pass gave up (flags 0x%x)", hs.flags);
    return DWCU_SUCCESS;
}

// ---- the R2C transform of fft3d on caller-provided device memory (used by
// noalloc.cu): sizes of the pieces it needs, then the transform itself
int fft3d_scratch_sizes(long long M, long long N, long long P, size_t *spec_bytes, size_t *real_bytes)
{
    if (M < 2 || N < 1 || P < 1 || (M % 2)) return fail(DWCU_ERROR_INVALID_VALUE, "M must be even and >= 2");
    if (!find_x((int) (M / 2)) || (N > 1 && !find_lines((int) N)) || !find_lines((int) P))
        return fail(DWCU_ERROR_UNSUPPORTED, "unsupported transform size %lld x %lld x %lld", M, N, P);
    const long long XP = (M + 3) & ~3LL, NKB = (M / 2 + 1 + KB - 1) / KB;
    *spec_bytes = align256(sizeof(float2) * (size_t) (NKB * N * KB * P + 8 * KB));
    *real_bytes = align256(sizeof(float) * (size_t) (XP * N * P + XP));
    return DWCU_SUCCESS;
}

static_assert(sizeof(JobScalars) <= 256, "noalloc.cu reserves 256 bytes for the scalars");

// S (spec_bytes), real (real_bytes) and sc must be zero on entry; tw holds
// the twiddle tables of the lengths M, M/2, N, P.  Enqueues on `stream`,
// waits for it and reports a bounded-wait timeout of any pass.
int fft3d_r2c_scratch(const float *d_in, long long M, long long N, long long P, float *d_out, cudaStream_t stream,
                      float2 *S, float *real, JobScalars *sc, const float2 *const tw[4])
{
    dwcu_job jj{};
    dwcu_job *j = &jj;
    dwcu_opts_init(&j->s);
    Geometry &g = j->g;
    g.M = M; g.N = N; g.P = P; g.pM = g.pN = g.pP = 1;
    g.wM = g.X = M; g.wN = g.Y = N; g.wP = g.Z = P;
    g.xp = find_x((int) (M / 2));
    g.yp = N > 1 ? find_lines((int) N) : nullptr;
    g.zp = find_lines((int) P);
    g.ytp = N > 1 ? find_y((int) N) : nullptr;
    if (!g.xp || (N > 1 && !g.yp) || !g.zp)
        return fail(DWCU_ERROR_UNSUPPORTED, "unsupported transform size %lld x %lld x %lld", M, N, P);
    g.XP = (M + 3) & ~3LL;
    g.NKB = (M / 2 + 1 + KB - 1) / KB;
    g.GP = (M + 3) & ~3LL;
    j->s.metric = DWCU_METRIC_IDIV;
    j->s.positivity = 1;
    j->stream = stream;
    j->nxb = x_blocks(g);
    j->tw_x = tw[0];
    j->tw_l = tw[1];
    j->tw_y = tw[2];
    j->tw_z = tw[3];
    j->S = S;
    j->sc = sc;
    const long long H = M / 2 + 1;
    const long long nspec = H * N * P;
    const int fb = (int) std::min<long long>(148 * 16, (nspec + 255) / 256);
    int rc = DWCU_SUCCESS;
    if (cudaMemcpy2DAsync(real, sizeof(float) * g.XP, d_in, sizeof(float) * M, sizeof(float) * M, N * P,
                          cudaMemcpyDeviceToDevice, stream) != cudaSuccess)
        rc = fail(DWCU_ERROR_CUDA, "copy failed");
    if (rc == DWCU_SUCCESS) rc = pass_x(j, XOP_FWD_COPY, 1, j->S, real, nullptr, nullptr, 0, 0);
    if (rc == DWCU_SUCCESS) rc = pass_y(j, LINES_FWD, j->S);
    if (rc == DWCU_SUCCESS) rc = pass_z(j, LINES_FWD, j->S);
    if (rc == DWCU_SUCCESS) {
        k_spec_unpack<<<fb, 256, 0, stream>>>(j->S, (int) H, (int) N, (int) P, (int) g.NKB,
                                               reinterpret_cast<float2 *>(d_out));
        ++g_launches;
        if (cudaGetLastError() != cudaSuccess) rc = fail(DWCU_ERROR_CUDA, "unpack launch failed");
    }
    cudaError_t e = cudaStreamSynchronize(stream);
    JobScalars hs{};
    if (e == cudaSuccess) e = cudaMemcpy(&hs, sc, sizeof hs, cudaMemcpyDeviceToHost);
    j->stream = nullptr;
    if (rc != DWCU_SUCCESS) return rc;
    if (e != cudaSuccess) return fail(DWCU_ERROR_CUDA, "transform failed: %s", cudaGetErrorString(e));
    if (hs.flags & ~3) return fail(DWCU_ERROR_TIMEOUT, "a bounded wait in a pass gave up (flags 0x%x)", hs.flags);
    return DWCU_SUCCESS;
}

}  // namespace dwcu

// ================================================================ C ABI

using namespace dwcu;

extern "C" {

void dwcu_opts_init(dwcu_opts *s)
{
    if (!s) return;
    memset(s, 0, sizeof *s);
    s->method = DWCU_METHOD_SHB;
    s->n_iter = 1;
    s->iter_type = DWCU_ITER_REL;
    s->maxiter = 250;
    s->err_rel = 0.02f;
    s->err_abs = 1.0f;
    s->bg = 1e-2f;
    s->bg_auto = 1;
    s->positivity = 1;
    s->border_quality = 2;
    s->start_condition = DWCU_START_FLAT;
    s->metric = DWCU_METRIC_IDIV;
    s->alphamax = 1.0f;
    s->device = 0;
    s->verbosity = 0;
    s->use_graph = 1;
}

int dwcu_deconvolve(const float *im, int64_t M, int64_t N, int64_t P, const float *psf, int64_t pM, int64_t pN,
                    int64_t pP, dwcu_opts *s, float *out)
{
    return one_call(im, M, N, P, psf, pM, pN, pP, s, out, false, nullptr);
}

int dwcu_deconvolve_device(const float *d_im, int64_t M, int64_t N, int64_t P, const float *d_psf, int64_t pM,
                           int64_t pN, int64_t pP, dwcu_opts *s, float *d_out, void *stream)
{
    return one_call(d_im, M, N, P, d_psf, pM, pN, pP, s, d_out, true, (cudaStream_t) stream);
}

int dwcu_plan_size(int64_t M, int64_t N, int64_t P, int64_t pM, int64_t pN, int64_t pP, int32_t border_quality,
                   int32_t method, int64_t work[3], int64_t *device_bytes)
{
    Geometry g;
    int rc = make_geometry(M, N, P, pM, pN, pP, border_quality, g);
    if (rc != DWCU_SUCCESS) return rc;
    if (work) { work[0] = g.X; work[1] = g.Y; work[2] = g.Z; }
    dwcu_opts s;
    dwcu_opts_init(&s);
    s.border_quality = border_quality;
    s.method = method;
    if (device_bytes) *device_bytes = job_bytes_estimate(g, s);
    return DWCU_SUCCESS;
}

int dwcu_job_create(int64_t M, int64_t N, int64_t P, int64_t pM, int64_t pN, int64_t pP, const dwcu_opts *s,
                    dwcu_job **job)
{
    if (!job) return fail(DWCU_ERROR_INVALID_VALUE, "job is NULL");
    return job_create(M, N, P, pM, pN, pP, s, job);
}

int dwcu_job_setup(dwcu_job *job, const float *im, const float *psf, int32_t on_device)
{
    if (!job || !im || !psf) return fail(DWCU_ERROR_INVALID_VALUE, "NULL argument");
    return job_setup(job, im, psf, on_device != 0);
}

int dwcu_job_step(dwcu_job *job, int32_t n, int32_t *remaining)
{
    if (!job) return fail(DWCU_ERROR_INVALID_VALUE, "job is NULL");
    return job_step(job, n, remaining);
}

int dwcu_batch_run(dwcu_job **jobs, int32_t n, void *stream)
{
    if (!jobs && n > 0) return fail(DWCU_ERROR_INVALID_VALUE, "jobs is NULL");
    return batch_run(jobs, n, (cudaStream_t) stream);
}

int dwcu_job_done(const dwcu_job *job) { return job && job->finished ? 1 : 0; }

int dwcu_job_result(dwcu_job *job, float *out, int32_t out_on_device, dwcu_opts *s_out)
{
    if (!job || !out) return fail(DWCU_ERROR_INVALID_VALUE, "NULL argument");
    return job_result(job, out, out_on_device != 0, s_out);
}

int dwcu_release_cache(int32_t device)
{
    std::vector<Block *> drop;
    {
        std::lock_guard<std::mutex> lk(g_blk_mu);
        for (auto &kv : g_blk_free) {
            if (device >= 0 && kv.first != device) continue;
            drop.insert(drop.end(), kv.second.begin(), kv.second.end());
            kv.second.clear();
        }
    }
    int cur = 0;
    const bool had = cudaGetDevice(&cur) == cudaSuccess;
    for (auto *b : drop) {
        cudaSetDevice(b->device);
        block_free(b);
    }
    if (had && !drop.empty()) cudaSetDevice(cur);  // the caller's current device as it was
    return DWCU_SUCCESS;
}

void dwcu_job_destroy(dwcu_job *j)
{
    if (!j) return;
    cudaSetDevice(j->s.device);
    if (j->stream) cudaStreamSynchronize(j->stream);
    check_guards(j);
    if (j->graph) cudaGraphExecDestroy(j->graph);
    if (j->block) block_put(j->block);
    if (j->ev0) cudaEventDestroy(j->ev0);
    if (j->ev1) cudaEventDestroy(j->ev1);
    if (j->ev2) cudaEventDestroy(j->ev2);
    for (auto e : j->ev_rb)
        if (e) cudaEventDestroy(e);
    if (j->h_err) cudaFreeHost(j->h_err);
    delete j;
}

int dwcu_job_set_stream(dwcu_job *job, void *stream)
{
    if (!job) return fail(DWCU_ERROR_INVALID_VALUE, "job is NULL");
    job->stream = stream ? (cudaStream_t) stream : job->ctx->stream;
    return DWCU_SUCCESS;
}

int64_t dwcu_job_bytes(const dwcu_job *job) { return job ? (int64_t) job->bytes : 0; }

// Between iterations a job's state is x_k (xa), x_{k-1} (xb, SHB), the error
// trace and the stopping rule's counters; the spectrum is recomputed from
// the estimates when the job continues (iter_input), and everything else
// (image, OTF, weights, scalars) by its set-up.
int dwcu_job_snapshot(dwcu_job *j, float *x, float *x_prev, float *trace, int32_t trace_capacity,
                      dwcu_job_state *st)
{
    if (!j || !st) return fail(DWCU_ERROR_INVALID_VALUE, "NULL argument");
    if (!j->setup_done) return fail(DWCU_ERROR_INVALID_VALUE, "snapshot before setup");
    memset(st, 0, sizeof *st);
    st->volume_elems = j->g.real_elems();
    st->next_iter = j->finished ? -1 : j->k_next;
    st->done_iters = j->done_iters;
    st->iter = j->it.iter;
    st->error = j->it.error;
    st->lasterror = j->it.lasterror;
    st->bg = j->s.bg;
    if (!x) return DWCU_SUCCESS;
    const bool shb = (j->s.method == DWCU_METHOD_SHB);
    if (shb && !x_prev) return fail(DWCU_ERROR_INVALID_VALUE, "an SHB snapshot needs x_prev");
    CU(cudaSetDevice(j->s.device));
    const size_t R = sizeof(float) * (size_t) st->volume_elems;
    CU(cudaMemcpyAsync(x, j->xa, R, cudaMemcpyDeviceToHost, j->stream));
    if (shb) CU(cudaMemcpyAsync(x_prev, j->xb, R, cudaMemcpyDeviceToHost, j->stream));
    const int ne = std::min(j->done_iters, std::max(0, (int) trace_capacity));
    if (trace && ne > 0) CU(cudaMemcpyAsync(trace, j->err, sizeof(float) * ne, cudaMemcpyDeviceToHost, j->stream));
    CU(cudaStreamSynchronize(j->stream));
    return DWCU_SUCCESS;
}

int dwcu_job_restore(dwcu_job *j, const float *x, const float *x_prev, const float *trace, const dwcu_job_state *st)
{
    if (!j || !x || !st) return fail(DWCU_ERROR_INVALID_VALUE, "NULL argument");
    if (!j->setup_done) return fail(DWCU_ERROR_INVALID_VALUE, "restore before setup");
    const bool shb = (j->s.method == DWCU_METHOD_SHB);
    if (shb && !x_prev) return fail(DWCU_ERROR_INVALID_VALUE, "an SHB snapshot needs x_prev");
    if (st->volume_elems != j->g.real_elems())
        return fail(DWCU_ERROR_INVALID_VALUE, "the snapshot is of a job of another size");
    if (st->bg != j->s.bg) return fail(DWCU_ERROR_INVALID_VALUE, "the snapshot's background differs from the job's");
    if (st->done_iters < 0 || st->done_iters > trace_cap(j->s) || st->next_iter < -1 ||
        st->next_iter >= j->it.niter || (st->next_iter >= 0 && st->next_iter != st->done_iters))
        return fail(DWCU_ERROR_INVALID_VALUE, "inconsistent iteration state (next %d, done %d)", st->next_iter,
                    st->done_iters);
    if (st->done_iters > 0 && !trace) return fail(DWCU_ERROR_INVALID_VALUE, "the error trace is missing");
    CU(cudaSetDevice(j->s.device));
    const size_t R = sizeof(float) * (size_t) st->volume_elems;
    CU(cudaMemcpyAsync(j->xa, x, R, cudaMemcpyHostToDevice, j->stream));
    if (shb) CU(cudaMemcpyAsync(j->xb, x_prev, R, cudaMemcpyHostToDevice, j->stream));
    if (st->done_iters > 0)
        CU(cudaMemcpyAsync(j->err, trace, sizeof(float) * st->done_iters, cudaMemcpyHostToDevice, j->stream));
    CU(cudaStreamSynchronize(j->stream));
    for (int i = 0; i < st->done_iters; ++i) j->trace[(size_t) i] = trace[i];
    j->done_iters = st->done_iters;
    j->k_next = st->next_iter;
    j->finished = st->next_iter < 0;
    j->it.iter = st->iter;
    j->it.error = st->error;
    j->it.lasterror = st->lasterror;
    j->spectrum_ready = false;
    j->spec = -1;
    return DWCU_SUCCESS;
}

const char *dwcu_last_error(void) { return g_last_error.c_str(); }
int dwcu_abi_version(void) { return DWCU_ABI_VERSION; }

int dwcu_tune_run(int32_t device, int32_t kind, int32_t n)
{
    if (kind < DWCU_PLAN_LINES || kind > DWCU_PLAN_X) return fail(DWCU_ERROR_INVALID_VALUE, "bad plan kind");
    if (tune_plan_count(kind, n) < 1) return fail(DWCU_ERROR_UNSUPPORTED, "no plan of length %d for this pass", n);
    DeviceCtx *ctx = nullptr;
    TRY(get_ctx(device, &ctx));
    CU(cudaSetDevice(device));
    int rc = DWCU_SUCCESS;
    tuned_choice(ctx, kind, n, &rc);
    return rc;
}
int dwcu_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}
int64_t dwcu_launch_count(void) { return g_launches; }

}  // extern "C"

namespace dwcu {
// The bounded-wait path of the passes (wait_all), exercised on its own: one
// block waits on an mbarrier phase that only completes when `arrive` is set
// (no copy is ever issued, so nothing is in flight when the block leaves).
__global__ void k_wait_selftest(int *err, unsigned polls, int arrive)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (arrive && threadIdx.x == 0) mbar_arrive(&bar);
    wait_all(&bar, 0, err, 1 << 8, polls);
}
}  // namespace dwcu

extern "C" {

int dwcu_debug_guards(int32_t mode)
{
    if (mode < 0 || mode > 2) return fail(DWCU_ERROR_INVALID_VALUE, "guard mode must be 0, 1 or 2");
    g_guard_mode.store(mode);
    return DWCU_SUCCESS;
}

int64_t dwcu_debug_guard_violations(void) { return g_guard_violations.load(); }

int dwcu_selftest_bounded_wait(int32_t device, int32_t arrive, uint32_t polls)
{
    if (polls < 1) return fail(DWCU_ERROR_INVALID_VALUE, "polls must be positive");
    DeviceCtx *ctx = nullptr;
    TRY(get_ctx(device, &ctx));
    CU(cudaSetDevice(device));
    int *d_flag = nullptr;
    CU(cudaMalloc(&d_flag, sizeof(int)));
    int h_flag = 0;
    cudaError_t e = cudaMemsetAsync(d_flag, 0, sizeof(int), ctx->stream);
    if (e == cudaSuccess) {
        k_wait_selftest<<<1, 64, 0, ctx->stream>>>(d_flag, polls, arrive ? 1 : 0);
        ++g_launches;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_flag, d_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(d_flag);
    if (e != cudaSuccess) return fail(DWCU_ERROR_CUDA, "bounded-wait self-test failed: %s", cudaGetErrorString(e));
    if (h_flag & ~0xff) return fail(DWCU_ERROR_TIMEOUT, "a bounded wait gave up after %u polls", polls);
    return DWCU_SUCCESS;
}

int dwcu_profile_enable(int32_t on)
{
    std::lock_guard<std::mutex> lk(g_prof_mu);
    g_prof_on = on != 0;
    return DWCU_SUCCESS;
}

int dwcu_profile_collect(dwcu_kernel_stat *stats, int32_t capacity, int32_t *count)
{
    std::lock_guard<std::mutex> lk(g_prof_mu);
    std::vector<double> ms(g_prof_classes.size(), 0.0);
    std::vector<long long> n(g_prof_classes.size(), 0);
    for (auto &r : g_prof_recs) {
        if (cudaEventSynchronize(r.b) != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        float t = 0.f;
        if (cudaEventElapsedTime(&t, r.a, r.b) == cudaSuccess) {
            ms[(size_t) r.cls] += t;
            n[(size_t) r.cls] += 1;
        } else {
            cudaGetLastError();
        }
        if (!r.owned_by_graph) {
            g_prof_pool.push_back(r.a);
            g_prof_pool.push_back(r.b);
        }
    }
    g_prof_recs.clear();
    int k = 0;
    for (size_t i = 0; i < g_prof_classes.size(); ++i) {
        if (n[i] == 0) continue;
        if (stats && k < capacity) {
            memset(&stats[k], 0, sizeof stats[k]);
            snprintf(stats[k].name, sizeof stats[k].name, "%s", g_prof_classes[i].name.c_str());
            stats[k].launches = n[i];
            stats[k].milliseconds = ms[i];
            stats[k].bytes_per_launch = g_prof_classes[i].bytes;
        }
        ++k;
    }
    if (count) *count = k;
    return DWCU_SUCCESS;
}

int dwcu_fft_r2c(const float *d_in, int64_t M, int64_t N, int64_t P, float *d_out, int32_t device, void *stream)
{
    return fft3d(d_in, M, N, P, d_out, device, (cudaStream_t) stream, true);
}

int dwcu_fft_c2r(const float *d_in, int64_t M, int64_t N, int64_t P, float *d_out, int32_t device, void *stream)
{
    return fft3d(d_in, M, N, P, d_out, device, (cudaStream_t) stream, false);
}

}  // extern "C"

// one image over several GPUs (slabs of z planes)
#include "slab.cuh"
