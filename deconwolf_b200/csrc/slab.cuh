// slab.cuh -- one image over several GPUs: the SHB / RL job split by z planes.
//
// Compiled as part of engine.cu (it drives the engine's passes).  For volumes
// whose job does not fit one GPU's memory; deconwolf itself handles those by
// tiling (src/dw.c:2001-2229), which changes the result at tile seams, while
// this split gives the whole-image result.
//
// Layout.  Part p of n holds the z planes z = l*n + p (l = 0, 1, ...): its
// real volumes, image planes and spectrum planes, in the whole job's layout
// with Zl = ceil((Z - p) / n) planes.  The image planes z < P of a part are
// its first Pl = ceil((P - p) / n) planes, so the x pass's image test and the
// pruned y passes run on a part unchanged, and every part holds about the
// same share of the image planes (the pruned passes stay balanced).  The x
// and y passes need nothing from other parts.  The z pass needs whole z
// lines: part p transforms the columns [c0, c0 + nc) of every plane (a
// plane's NKB*Y*KB complex elements, nc a multiple of KB).  Where every pair
// of the parts' GPUs has peer access (always, for parts on one GPU), the z
// pass reads and writes those columns where they lie, through a table of
// the Z planes' addresses (k_lines' planes mode: one kernel does the
// transform and the exchange, the NVLink transfer overlapping the FFT
// arithmetic block by block).  Otherwise the columns are gathered into a
// column buffer T ([Z][nc], plane z at z*nc) by one pitched copy from each
// part (part q's planes are the rows q, q+n, ... of T), transformed there,
// and scattered back the same way (copy engines; staged through the host
// where the GPUs have no peer access).  The OTF of the part's columns stays
// with the part ([Z][nc]).
//
// Order between parts (slab_barrier): before the z pass, every part's y pass
// is complete; before the y pass after it, every part's z pass (or scatter)
// is complete.  Parts driven by one process: each part records an event and
// waits on every other part's.  One process per part (dwcu_slab_part_*): the
// caller's barrier, a stream-ordered collective such as an NCCL all-reduce,
// and the peers' spectra mapped through CUDA IPC handles.  During a z pass,
// part p reads and writes only its own columns, which no other part touches.
//
// Supported: SHB and RL, every stopping rule, every start (the low-pass
// start smooths the whole image on part 0's GPU and deals its planes out),
// every border quality, and periodic margins along x and y (rows within a
// part's planes).  Not supported: periodic margins along z (a z length
// without an exact-size transform at border_quality 0 / 1: the margin planes
// would be copies of other parts' planes).

struct dwcu_slab;

namespace dwcu {

struct SlabPart {
    dwcu_job *j = nullptr;         // the part's job: planes z = l*n + p
    int device = -1;
    long long zl = 0, pl = 0;      // planes, image planes
    long long c0 = 0, nc = 0;      // z-pass columns [c0, c0 + nc) of a plane
    cudaStream_t stream = nullptr;
    cudaEvent_t ev = nullptr;      // ordering between parts
    double *psum = nullptr;        // per iteration: the error sum of the part's tiles
    float2 **planes = nullptr;     // planes mode: the address of every plane z (on this part's GPU)
    float2 *S = nullptr;           // the part's spectrum planes (its own, or mapped from another process)
    void *ipc_base = nullptr;      // the mapped allocation of another process's part
};

// the planes and z-pass columns of part p of n (host arithmetic only)
static void slab_layout(long long Z, long long P, long long cols, int n, int p, long long *zl, long long *pl,
                        long long *c0, long long *nc)
{
    *zl = Z > p ? (Z - p + n - 1) / n : 0;
    *pl = P > p ? (P - p + n - 1) / n : 0;
    const long long units = cols / KB;
    const long long u0 = units * p / n, u1 = units * (p + 1) / n;
    *c0 = u0 * KB;
    *nc = (u1 - u0) * KB;
}

// k_psf_embed restricted to one part's planes: the PSF voxel that lands on
// plane z goes to local plane z / n when z % n == p
__global__ void k_slab_psf_embed(const float *__restrict__ psf, int pM, int pN, int pP, const long long *amax,
                                 float *__restrict__ dst, int X, int Y, int Z, int XP, float scale, int n, int p)
{
    const long long cnt = (long long) pM * pN * pP;
    const long long am = *amax;
    const int ac = (int) (am / ((long long) pM * pN));
    const int ab = (int) ((am - (long long) ac * pM * pN) / pM);
    const int aa = (int) (am - (long long) ac * pM * pN - (long long) ab * pM);
    for (long long k = blockIdx.x * (long long) blockDim.x + threadIdx.x; k < cnt;
         k += (long long) gridDim.x * blockDim.x) {
        const int c = (int) (k / ((long long) pM * pN));
        const int b = (int) ((k - (long long) c * pM * pN) / pM);
        const int a = (int) (k - (long long) c * pM * pN - (long long) b * pM);
        int z = (c - ac) % Z; if (z < 0) z += Z;
        if (z % n != p) continue;
        int x = (a - aa) % X; if (x < 0) x += X;
        int y = (b - ab) % Y; if (y < 0) y += Y;
        dst[((long long) (z / n) * Y + y) * XP + x] = psf[k] * scale;
    }
}

// the sum of a part's tile partials, in the fixed order of k_err_final
__global__ void __launch_bounds__(kRedThreads) k_slab_err_sum(const double *__restrict__ part, int nb, double *out)
{
    __shared__ double s[kRedThreads];
    double v = 0.0;
    for (int i = threadIdx.x; i < nb; i += kRedThreads) v += part[i];
    s[threadIdx.x] = v;
    __syncthreads();
    for (int o = kRedThreads / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = s[0];
}

// the parts' sums in part order: the iteration's error value
__global__ void k_slab_err_combine(const double *__restrict__ sums, int n, double count, float *err_out)
{
    if (threadIdx.x != 0) return;
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += sums[i];
    *err_out = (float) (s / count);
}

}  // namespace dwcu

struct dwcu_slab {
    dwcu_opts s;
    dwcu::Geometry g;              // the whole job
    std::vector<dwcu::SlabPart> parts;
    double *sums = nullptr;        // on part 0's device: the parts' error sums of one iteration
    bool copies = false;           // z pass on gathered copies instead of in place
    int local = -1;                // one process per part: the part this process holds (-1: all)
    dwcu_slab_sync sync{};         // ... and the caller's collectives
    double *sync_buf = nullptr;    // ... on a device buffer of the caller's
    // the part that times the run and holds the error trace: part 0, or the
    // process's own part
    dwcu::SlabPart &lead() { return parts[(size_t) (local >= 0 ? local : 0)]; }
    dwcu::Iter it;
    int k_next = -1;
    bool spectrum_ready = false;
    int done_iters = 0;
    bool finished = false;
    bool setup_done = false;
};

namespace dwcu {

static void slab_destroy(dwcu_slab *sl)
{
    if (!sl) return;
    for (auto &pt : sl->parts)
        if (pt.stream) {
            cudaSetDevice(pt.device);
            cudaStreamSynchronize(pt.stream);
        }
    for (auto &pt : sl->parts)
        if (pt.ipc_base) {
            cudaSetDevice(sl->lead().device);
            cudaIpcCloseMemHandle(pt.ipc_base);
        }
    for (auto &pt : sl->parts) {
        if (pt.device < 0) continue;
        cudaSetDevice(pt.device);
        if (pt.j) dwcu_job_destroy(pt.j);
        if (pt.psum) cudaFree(pt.psum);
        if (pt.planes) cudaFree(pt.planes);
        if (pt.ev) cudaEventDestroy(pt.ev);
        if (pt.stream) cudaStreamDestroy(pt.stream);
    }
    if (sl->sums && !sl->parts.empty()) {
        cudaSetDevice(sl->parts[0].device);
        cudaFree(sl->sums);
    }
    cudaGetLastError();
    delete sl;
}

static int slab_part_create(dwcu_slab *sl, int p, int device)
{
    const Geometry &g = sl->g;
    const int n = (int) sl->parts.size();
    SlabPart &pt = sl->parts[(size_t) p];
    slab_layout(g.Z, g.P, g.NKB * g.Y * KB, n, p, &pt.zl, &pt.pl, &pt.c0, &pt.nc);
    DeviceCtx *ctx = nullptr;
    TRY(get_ctx(device, &ctx));
    pt.device = device;
    CU(cudaSetDevice(device));
    CU(cudaStreamCreateWithFlags(&pt.stream, cudaStreamNonBlocking));
    CU(cudaEventCreateWithFlags(&pt.ev, cudaEventDisableTiming));
    CU(cudaMalloc(&pt.psum, sizeof(double) * (size_t) trace_cap(sl->s)));
    dwcu_job *j = new dwcu_job();
    pt.j = j;
    j->s = sl->s;
    j->s.device = device;
    j->g = g;
    j->g.Z = pt.zl;
    j->g.P = pt.pl;
    j->ctx = ctx;
    j->stream = pt.stream;
    j->slab_elems = g.Z * pt.nc;
    j->slab_copies = sl->copies;
    TRY(alloc_job(j));
    pt.S = j->S;
    TRY(get_twiddles(ctx, g.X, &j->tw_x));
    TRY(get_twiddles(ctx, g.X / 2, &j->tw_l));
    if (g.Y > 1) TRY(get_twiddles(ctx, g.Y, &j->tw_y));
    TRY(get_twiddles(ctx, g.Z, &j->tw_z));
    if (cudaEventCreate(&j->ev0) != cudaSuccess || cudaEventCreate(&j->ev1) != cudaSuccess ||
        cudaEventCreate(&j->ev2) != cudaSuccess)
        return fail(DWCU_ERROR_CUDA, "event creation failed");
    j->trace.assign((size_t) trace_cap(sl->s), 0.f);
    return DWCU_SUCCESS;
}

static int slab_create(long long M, long long N, long long P, long long pM, long long pN, long long pP,
                       const dwcu_opts *s, int nparts, const int32_t *devices, dwcu_slab **out)
{
    *out = nullptr;
    if (!s) return fail(DWCU_ERROR_INVALID_VALUE, "opts is NULL");
    TRY(check_opts(*s));
    if (nparts < 1 || nparts > 64) return fail(DWCU_ERROR_INVALID_VALUE, "parts must be 1..64 (got %d)", nparts);
    Geometry g;
    TRY(make_geometry(M, N, P, pM, pN, pP, s->border_quality, g));
    if (g.wz)
        return fail(DWCU_ERROR_UNSUPPORTED, "job z size %lld needs periodic margins along z: not with parts", g.wP);
    if (nparts > g.Z) return fail(DWCU_ERROR_UNSUPPORTED, "%d parts for %lld z planes", nparts, g.Z);
    if (g.NKB * g.Y < nparts) return fail(DWCU_ERROR_UNSUPPORTED, "too few z-pass columns for %d parts", nparts);
    const int dev0 = devices ? devices[0] : s->device;
    DeviceCtx *ctx0 = nullptr;
    TRY(get_ctx(dev0, &ctx0));
    CU(cudaSetDevice(dev0));
    tune_geometry(ctx0, g);
    dwcu_slab *sl = new dwcu_slab();
    sl->s = *s;
    sl->g = g;
    sl->parts.resize((size_t) nparts);
    // the z pass in place needs peer access between every pair of the parts'
    // GPUs; DWCU_SLAB_TRANSPOSE=copy asks for the copies regardless
    const char *tr = getenv("DWCU_SLAB_TRANSPOSE");
    sl->copies = tr && strcmp(tr, "copy") == 0;
    for (int p = 0; p < nparts; ++p)
        for (int q = 0; q < nparts; ++q) {
            const int a = devices ? devices[p] : s->device, b = devices ? devices[q] : s->device;
            int can = 0;
            if (a != b && (cudaDeviceCanAccessPeer(&can, a, b) != cudaSuccess || !can)) sl->copies = true;
        }
    cudaGetLastError();
    int rc = DWCU_SUCCESS;
    for (int p = 0; p < nparts && rc == DWCU_SUCCESS; ++p) rc = slab_part_create(sl, p, devices ? devices[p] : s->device);
    // peer access between the parts' GPUs, where the devices allow it (the
    // copies work without it, staged through the host)
    for (int p = 0; p < nparts && rc == DWCU_SUCCESS; ++p)
        for (int q = 0; q < nparts; ++q) {
            const int a = sl->parts[(size_t) p].device, b = sl->parts[(size_t) q].device;
            int can = 0;
            if (a == b || cudaDeviceCanAccessPeer(&can, a, b) != cudaSuccess || !can) continue;
            cudaSetDevice(a);
            const cudaError_t e = cudaDeviceEnablePeerAccess(b, 0);
            if (e != cudaSuccess && e != cudaErrorPeerAccessAlreadyEnabled) rc = fail(DWCU_ERROR_CUDA, "peer access %d -> %d: %s", a, b, cudaGetErrorString(e));
            cudaGetLastError();
        }
    if (rc == DWCU_SUCCESS) {
        cudaSetDevice(dev0);
        if (cudaMalloc(&sl->sums, sizeof(double) * (size_t) nparts) != cudaSuccess)
            rc = fail(DWCU_ERROR_OUT_OF_MEMORY, "cudaMalloc of the error sums failed");
    }
    if (rc != DWCU_SUCCESS) {
        slab_destroy(sl);
        return rc;
    }
    *out = sl;
    return DWCU_SUCCESS;
}

// planes mode: each own part's table of the Z planes' addresses (once every
// part's spectrum is known)
static int slab_plane_tables(dwcu_slab *sl)
{
    if (sl->copies) return DWCU_SUCCESS;
    const Geometry &g = sl->g;
    const long long n = (long long) sl->parts.size();
    const long long plane = g.NKB * g.Y * KB;
    std::vector<float2 *> tab((size_t) g.Z);
    for (long long z = 0; z < g.Z; ++z) {
        float2 *S = sl->parts[(size_t) (z % n)].S;
        if (!S) return fail(DWCU_ERROR_INVALID_VALUE, "part %lld's spectrum is not mapped (dwcu_slab_part_import)", z % n);
        tab[(size_t) z] = S + (z / n) * plane;
    }
    for (auto &pt : sl->parts) {
        if (!pt.j || pt.planes) continue;
        CU(cudaSetDevice(pt.device));
        CU(cudaMalloc(&pt.planes, sizeof(float2 *) * (size_t) g.Z));
        CU(cudaMemcpy(pt.planes, tab.data(), sizeof(float2 *) * (size_t) g.Z, cudaMemcpyHostToDevice));
    }
    return DWCU_SUCCESS;
}

// the caller's collectives (one process per part)
static int slab_sync_barrier(dwcu_slab *sl)
{
    SlabPart &me = sl->lead();
    CU(cudaSetDevice(me.device));
    if (sl->sync.barrier(sl->sync.ctx, (void *) me.stream) != 0)
        return fail(DWCU_ERROR_INTERNAL, "the caller's barrier failed");
    return DWCU_SUCCESS;
}
static int slab_sync_allreduce(dwcu_slab *sl, int n, int op)
{
    SlabPart &me = sl->lead();
    CU(cudaSetDevice(me.device));
    if (sl->sync.allreduce(sl->sync.ctx, (void *) me.stream, n, op) != 0)
        return fail(DWCU_ERROR_INTERNAL, "the caller's all-reduce failed");
    return DWCU_SUCCESS;
}

// every part waits until every other part has reached this point
static int slab_barrier(dwcu_slab *sl)
{
    if (sl->local >= 0) return slab_sync_barrier(sl);
    if (sl->parts.size() < 2) return DWCU_SUCCESS;
    for (auto &pt : sl->parts) {
        CU(cudaSetDevice(pt.device));
        CU(cudaEventRecord(pt.ev, pt.stream));
    }
    for (auto &pt : sl->parts) {
        CU(cudaSetDevice(pt.device));
        for (auto &q : sl->parts)
            if (&q != &pt) CU(cudaStreamWaitEvent(pt.stream, q.ev, 0));
    }
    return DWCU_SUCCESS;
}

// part 0 waits until every part has reached this point (one process per
// part: every part waits)
static int slab_join0(dwcu_slab *sl)
{
    if (sl->local >= 0) return slab_sync_barrier(sl);
    if (sl->parts.size() < 2) return DWCU_SUCCESS;
    for (size_t p = 1; p < sl->parts.size(); ++p) {
        CU(cudaSetDevice(sl->parts[p].device));
        CU(cudaEventRecord(sl->parts[p].ev, sl->parts[p].stream));
    }
    SlabPart &p0 = sl->parts[0];
    CU(cudaSetDevice(p0.device));
    for (size_t p = 1; p < sl->parts.size(); ++p) CU(cudaStreamWaitEvent(p0.stream, sl->parts[p].ev, 0));
    return DWCU_SUCCESS;
}

// part pt's columns of every part's planes l < (image_only ? pl : zl) into
// dst ([Z][nc]), or (scatter) back from T
static int slab_transpose(dwcu_slab *sl, SlabPart &pt, float2 *buf, bool image_only, bool scatter)
{
    const long long plane = sl->g.NKB * sl->g.Y * KB;
    const long long n = (long long) sl->parts.size();
    CU(cudaSetDevice(pt.device));
    for (long long q = 0; q < n; ++q) {
        SlabPart &o = sl->parts[(size_t) q];
        const long long h = image_only ? o.pl : o.zl;
        if (h == 0) continue;
        float2 *cols = buf + q * pt.nc;    // rows q, q+n, ... of [Z][nc]
        float2 *planes = o.S + pt.c0;      // the part's planes, this part's columns
        const size_t cp = sizeof(float2) * (size_t) (n * pt.nc), pp = sizeof(float2) * (size_t) plane;
        const size_t w = sizeof(float2) * (size_t) pt.nc;
        if (scatter)
            CU(cudaMemcpy2DAsync(planes, pp, cols, cp, w, (size_t) h, cudaMemcpyDefault, pt.stream));
        else
            CU(cudaMemcpy2DAsync(cols, cp, planes, pp, w, (size_t) h, cudaMemcpyDefault, pt.stream));
    }
    return DWCU_SUCCESS;
}

// z lines of the part's columns (planes >= nin read as zero, only planes < nout written)
static int slab_zpass(dwcu_slab *sl, SlabPart &pt, int mode, float2 *data, long long nin, long long nout)
{
    const Geometry &g = sl->g;
    CU(cudaSetDevice(pt.device));
    return launch_lines(pt.j, g.zp, pt.j->tw_z, g.Z, pt.nc, 0, 1, pt.nc, mode, data, "z", nin, nout);
}

// the spectrum times the OTF (conj: its conjugate) over all parts, in place;
// in_img: only the input's planes z < P are non-zero; out_img: only the
// result's planes z < P are needed (the pruning of conv_forward / conv_backward)
static int slab_conv(dwcu_slab *sl, int conj, bool in_img, bool out_img)
{
    const Geometry &g = sl->g;
    for (auto &pt : sl->parts) {
        if (!pt.j) continue;
        CU(cudaSetDevice(pt.device));
        const long long h = in_img ? pt.pl : pt.zl;
        if (h > 0) TRY(pass_y(pt.j, LINES_FWD, pt.j->S, h));
    }
    TRY(slab_barrier(sl));
    const int mode = conj ? LINES_CONV_CONJ : LINES_CONV;
    for (auto &pt : sl->parts) {
        if (!pt.j) continue;
        if (sl->copies) {
            TRY(slab_transpose(sl, pt, pt.j->T, in_img, false));
            TRY(slab_zpass(sl, pt, mode, pt.j->T, in_img ? g.P : g.Z, out_img ? g.P : g.Z));
            TRY(slab_transpose(sl, pt, pt.j->T, out_img, true));
        } else {
            CU(cudaSetDevice(pt.device));
            TRY(launch_lines(pt.j, g.zp, pt.j->tw_z, g.Z, pt.nc, 0, 1, pt.nc, mode, pt.j->K, "z", in_img ? g.P : g.Z,
                             out_img ? g.P : g.Z, pt.planes, pt.c0));
        }
    }
    TRY(slab_barrier(sl));
    for (auto &pt : sl->parts) {
        if (!pt.j) continue;
        CU(cudaSetDevice(pt.device));
        const long long h = out_img ? pt.pl : pt.zl;
        if (h > 0) TRY(pass_y(pt.j, LINES_INV, pt.j->S, h));
    }
    return DWCU_SUCCESS;
}

// The low-pass start (method_shb.c:278-285, method_rl.c:290-297): the image
// smoothed by fim_gsmooth (sigma 8) along x, y and z -- the z smoothing
// needs whole image columns, so the whole image is smoothed on one GPU
// (part 0's, or with one process per part each process's own; job_setup's
// kernels and taps) -- then each part's image planes are copied into the
// corner of its zeroed x_0.
static int slab_lowpass_start(dwcu_slab *sl, const float *im)
{
    if (sl->s.start_condition != DWCU_START_LP) return DWCU_SUCCESS;
    const Geometry &g = sl->g;
    const int n = (int) sl->parts.size();
    SlabPart &p0 = sl->lead();
    CU(cudaSetDevice(p0.device));
    const long long nimg = g.M * g.N * g.P;
    float *t = nullptr;
    CU(cudaMalloc(&t, sizeof(float) * (size_t) (2 * nimg)));
    float *t1 = t, *t2 = t + nimg;
    int rc = DWCU_SUCCESS;
    auto run = [&]() -> int {
        cudaStream_t st = p0.stream;
        const int gb = (int) std::min<long long>(148 * 16, (nimg + 255) / 256);
        GaussTaps K = gauss_taps(8.0f);
        CU(cudaMemcpyAsync(t2, im, sizeof(float) * (size_t) nimg, cudaMemcpyHostToDevice, st));
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
        CU(cudaEventRecord(p0.ev, st));
        for (int p = 0; p < n; ++p) {
            SlabPart &pt = sl->parts[(size_t) p];
            dwcu_job *j = pt.j;
            if (!j) continue;
            CU(cudaSetDevice(pt.device));
            if (&pt != &p0) CU(cudaStreamWaitEvent(pt.stream, p0.ev, 0));
            CU(cudaMemsetAsync(j->xa, 0, sizeof(float) * (size_t) j->g.real_elems(), pt.stream));
            for (long long l = 0; l < pt.pl; ++l) {
                const long long z = l * n + p;
                CU(cudaMemcpy2DAsync(j->xa + l * g.Y * g.XP, sizeof(float) * g.XP, lp + z * g.M * g.N,
                                     sizeof(float) * g.M, sizeof(float) * g.M, g.N, cudaMemcpyDefault, pt.stream));
            }
        }
        return DWCU_SUCCESS;
    };
    rc = run();
    // the work space is freed once every part's copies are done
    for (auto &pt : sl->parts) {
        if (!pt.j) continue;
        cudaSetDevice(pt.device);
        cudaStreamSynchronize(pt.stream);
    }
    cudaSetDevice(p0.device);
    cudaFree(t);
    return rc;
}

// image planes and PSF into the parts; statistics, OTF, weights and the start
// estimate (job_setup's steps, method_shb.c:108-296, over the parts)
static int slab_setup(dwcu_slab *sl, const float *im, const float *psf)
{
    PhaseRange pr("dwcu split setup");
    const Geometry &g = sl->g;
    const int n = (int) sl->parts.size();
    const long long npsf = g.pM * g.pN * g.pP;
    const unsigned long long wmnp = (unsigned long long) (g.wM * g.wN * g.wP);
    TRY(slab_plane_tables(sl));
    for (int p = 0; p < n; ++p) {
        SlabPart &pt = sl->parts[(size_t) p];
        dwcu_job *j = pt.j;
        if (!j) continue;
        CU(cudaSetDevice(pt.device));
        cudaStream_t st = pt.stream;
        if (&pt == &sl->lead()) CU(cudaEventRecord(j->ev0, st));
        for (long long l = 0; l < pt.pl; ++l) {
            const long long z = l * n + p;
            CU(cudaMemcpy2DAsync(j->gimg + l * g.N * g.GP, sizeof(float) * g.GP, im + z * g.M * g.N,
                                 sizeof(float) * g.M, sizeof(float) * g.M, g.N, cudaMemcpyHostToDevice, st));
        }
        CU(cudaMemcpyAsync(j->psf_dev, psf, sizeof(float) * npsf, cudaMemcpyHostToDevice, st));
        CU(cudaMemsetAsync(j->sc, 0, sizeof(JobScalars), st));
        if (pt.pl > 0) {
            const long long nrows = g.N * pt.pl;
            const long long rpb = (nrows + j->n_spart - 1) / j->n_spart;
            const int nsb = (int) ((nrows + rpb - 1) / rpb);
            k_stats_partial<<<nsb, kRedThreads, 0, st>>>(j->gimg, g.GP, (int) g.M, nrows, rpb, j->spart);
            CHECK_LAUNCH();
            k_stats_final<<<1, kRedThreads, 0, st>>>(j->spart, nsb, j->sc, j->s.bg_auto, j->s.bg, wmnp);
            CHECK_LAUNCH();
        }
        const long long per = (npsf + j->n_apart - 1) / j->n_apart;
        const int nab = (int) ((npsf + per - 1) / per);
        k_argmax_partial<<<nab, kRedThreads, 0, st>>>(j->psf_dev, npsf, per, j->apart, &j->sc->flags);
        CHECK_LAUNCH();
        k_argmax_final<<<1, 32, 0, st>>>(j->apart, nab, j->amax);
        CHECK_LAUNCH();
    }
    // the parts' statistics, combined in part order (k_stats_final's
    // formulas), go back to every part
    double sumg = 0.0;
    float gmin = INFINITY;
    int flags = 0;
    for (auto &pt : sl->parts) {
        if (!pt.j) continue;
        JobScalars hs{};
        CU(cudaSetDevice(pt.device));
        CU(cudaMemcpyAsync(&hs, pt.j->sc, sizeof hs, cudaMemcpyDeviceToHost, pt.stream));
        CU(cudaStreamSynchronize(pt.stream));
        flags |= hs.flags;
        if (pt.pl > 0) {
            sumg += hs.sumg;
            gmin = std::fmin(gmin, hs.gmin);
        }
    }
    if (sl->local >= 0) {
        // over the processes: the image sum and the parts with non-finite
        // image or PSF values added, the minimum taken
        SlabPart &me = sl->lead();
        double v[3] = {sumg, (double) (flags & 1), (double) ((flags >> 1) & 1)};
        CU(cudaSetDevice(me.device));
        CU(cudaMemcpyAsync(sl->sync_buf, v, sizeof v, cudaMemcpyHostToDevice, me.stream));
        TRY(slab_sync_allreduce(sl, 3, 0));
        CU(cudaMemcpyAsync(v, sl->sync_buf, sizeof v, cudaMemcpyDeviceToHost, me.stream));
        CU(cudaStreamSynchronize(me.stream));
        sumg = v[0];
        flags = (v[1] > 0 ? 1 : 0) | (v[2] > 0 ? 2 : 0);
        double m = (double) gmin;
        CU(cudaMemcpyAsync(sl->sync_buf, &m, sizeof m, cudaMemcpyHostToDevice, me.stream));
        TRY(slab_sync_allreduce(sl, 1, 1));
        CU(cudaMemcpyAsync(&m, sl->sync_buf, sizeof m, cudaMemcpyDeviceToHost, me.stream));
        CU(cudaStreamSynchronize(me.stream));
        gmin = (float) m;
    }
    if (flags & 1) return fail(DWCU_ERROR_INPUT, "the image contains non-finite values");
    if (flags & 2) return fail(DWCU_ERROR_INPUT, "the PSF contains non-finite values");
    if (g.wx || g.wy) {
        // the periodic margins assume the PSF maximum within h of both ends (as job_setup)
        long long am = 0;
        SlabPart &p0 = sl->lead();
        CU(cudaSetDevice(p0.device));
        CU(cudaMemcpy(&am, p0.j->amax, sizeof am, cudaMemcpyDeviceToHost));
        const long long ax = am % g.pM, ay = (am / g.pM) % g.pN;
        auto off = [](long long a, long long p) { return std::max(a, p - 1 - a); };
        if ((g.wx && off(ax, g.pM) > g.hx) || (g.wy && off(ay, g.pN) > g.hy))
            return fail(DWCU_ERROR_UNSUPPORTED,
                        "border_quality %d with a job size that has no exact transform needs the PSF maximum at "
                        "its centre (maximum at %lld, %lld of %lld x %lld)",
                        sl->s.border_quality, ax, ay, g.pM, g.pN);
    }
    JobScalars all{};
    all.gmin = gmin;
    all.sumg = sumg;
    all.bg = sl->s.bg_auto ? (gmin < 1e-2f ? 1e-2f : gmin) : sl->s.bg;
    all.x0 = (float) sumg / (float) wmnp;
    all.flags = 0;
    if (sl->s.bg_auto) sl->s.bg = all.bg;
    const float scale = (float) (1.0 / ((double) g.X * (double) g.Y * (double) g.Z));
    for (int p = 0; p < n; ++p) {
        SlabPart &pt = sl->parts[(size_t) p];
        dwcu_job *j = pt.j;
        if (!j) continue;
        CU(cudaSetDevice(pt.device));
        cudaStream_t st = pt.stream;
        CU(cudaMemcpyAsync(j->sc, &all, sizeof all, cudaMemcpyHostToDevice, st));
        CU(cudaStreamSynchronize(st));  // `all` is a host local
        j->s.bg = sl->s.bg;
        // the OTF: PSF planes of this part, x and y transforms here
        CU(cudaMemsetAsync(j->xb, 0, sizeof(float) * (size_t) j->g.real_elems(), st));
        k_slab_psf_embed<<<(int) std::min<long long>(4096, (npsf + 255) / 256), 256, 0, st>>>(
            j->psf_dev, (int) g.pM, (int) g.pN, (int) g.pP, j->amax, j->xb, (int) g.X, (int) g.Y, (int) g.Z,
            (int) g.XP, scale, n, p);
        CHECK_LAUNCH();
        TRY(pass_x(j, XOP_FWD_COPY, 1, j->S, j->xb, nullptr, nullptr, 0, 0, -1, false));
        TRY(pass_y(j, LINES_FWD, j->S));
    }
    // ... and the z transform of the part's columns, kept as its OTF
    TRY(slab_barrier(sl));
    for (auto &pt : sl->parts) {
        if (!pt.j) continue;
        TRY(slab_transpose(sl, pt, pt.j->K, false, false));
        TRY(slab_zpass(sl, pt, LINES_FWD, pt.j->K, g.Z, g.Z));
    }
    TRY(slab_barrier(sl));  // every gather has read the spectra before they change

    // Bertero weights: W = 1/P1 where P1 = K^T 1_image > 0.01 (method_shb.c:216-235)
    if (sl->lead().j->W) {
        for (auto &pt : sl->parts) {
            if (!pt.j) continue;
            CU(cudaSetDevice(pt.device));
            TRY(pass_x(pt.j, XOP_FWD_ONES, 1, pt.j->S, nullptr, nullptr, nullptr, 0, 0));
        }
        TRY(slab_conv(sl, 1, false, false));
        for (auto &pt : sl->parts) {
            if (!pt.j) continue;
            CU(cudaSetDevice(pt.device));
            TRY(pass_x(pt.j, XOP_WEIGHTS, 0, pt.j->S, nullptr, nullptr, pt.j->W, 0, 0));
        }
    }
    // start estimate (method_shb.c:264-276); x_{-1} = x_0
    TRY(slab_lowpass_start(sl, im));
    for (auto &pt : sl->parts) {
        dwcu_job *j = pt.j;
        if (!j) continue;
        CU(cudaSetDevice(pt.device));
        cudaStream_t st = pt.stream;
        const long long nv = j->g.real_elems();
        const size_t R = sizeof(float) * (size_t) nv;
        const int fb = (int) std::min<long long>(148 * 16, (nv + 255) / 256);
        if (sl->s.start_condition == DWCU_START_FLAT) {
            k_fill_scalar<<<fb, 256, 0, st>>>(j->xa, nv, j->sc);
            CHECK_LAUNCH();
        } else if (sl->s.start_condition == DWCU_START_IDENTITY) {
            CU(cudaMemsetAsync(j->xa, 0, R, st));
            if (pt.pl > 0) {
                k_embed_image<<<fb, 256, 0, st>>>(j->gimg, g.GP, (int) g.M, (int) g.N, (int) pt.pl, j->xa, (int) g.XP,
                                                  (int) g.Y);
                CHECK_LAUNCH();
            }
        }
        if (sl->s.method == DWCU_METHOD_SHB) CU(cudaMemcpyAsync(j->xb, j->xa, R, cudaMemcpyDeviceToDevice, st));
    }
    sl->it.init(sl->s);
    sl->k_next = sl->it.next();
    sl->finished = (sl->k_next < 0);
    sl->spectrum_ready = false;
    sl->done_iters = 0;
    sl->setup_done = true;
    TRY(slab_join0(sl));
    CU(cudaSetDevice(sl->lead().device));
    CU(cudaEventRecord(sl->lead().j->ev1, sl->lead().stream));
    return DWCU_SUCCESS;
}

// iteration k's input transform (iter_input on every part)
static int slab_input(dwcu_slab *sl, int k)
{
    for (auto &pt : sl->parts) {
        if (!pt.j) continue;
        CU(cudaSetDevice(pt.device));
        TRY(iter_input(pt.j, k));
    }
    return DWCU_SUCCESS;
}

// forward half of iteration k (iter_forward over the parts): y = K p_k,
// error_k on part 0 (with one process per part: on every part, from the
// caller's all-reduce of the parts' sums); with `ratio`, the ratio's transform
static int slab_forward(dwcu_slab *sl, int k, bool ratio)
{
    const Geometry &g = sl->g;
    const bool shb = (sl->s.method == DWCU_METHOD_SHB);
    TRY(slab_conv(sl, 0, false, true));
    const int op = ratio ? (shb ? XOP_RATIO_SHB : XOP_RATIO_RL) : XOP_ERROR_ONLY;
    const long long ytiles = (g.Y + g.xp->R - 1) / g.xp->R;
    for (auto &pt : sl->parts) {
        if (!pt.j) continue;
        CU(cudaSetDevice(pt.device));
        const long long tiles = (op == XOP_RATIO_RL) ? pt.j->nxb : pt.pl * ytiles;
        if (tiles > 0) TRY(pass_x(pt.j, op, ratio ? 1 : 0, pt.j->S, nullptr, nullptr, nullptr, 0, 0, tiles));
        k_slab_err_sum<<<1, kRedThreads, 0, pt.stream>>>(pt.j->partial, (int) tiles, pt.psum + k);
        CHECK_LAUNCH();
    }
    if (sl->local >= 0) {
        SlabPart &me = sl->lead();
        CU(cudaSetDevice(me.device));
        CU(cudaMemcpyAsync(sl->sync_buf, me.psum + k, sizeof(double), cudaMemcpyDeviceToDevice, me.stream));
        TRY(slab_sync_allreduce(sl, 1, 0));
        k_slab_err_combine<<<1, 32, 0, me.stream>>>(sl->sync_buf, 1, (double) (g.M * g.N * g.P), me.j->err + k);
        CHECK_LAUNCH();
        return DWCU_SUCCESS;
    }
    TRY(slab_join0(sl));
    SlabPart &p0 = sl->parts[0];
    CU(cudaSetDevice(p0.device));
    for (size_t q = 0; q < sl->parts.size(); ++q)
        CU(cudaMemcpyAsync(sl->sums + q, sl->parts[q].psum + k, sizeof(double), cudaMemcpyDefault, p0.stream));
    k_slab_err_combine<<<1, 32, 0, p0.stream>>>(sl->sums, (int) sl->parts.size(), (double) (g.M * g.N * g.P),
                                                p0.j->err + k);
    CHECK_LAUNCH();
    return DWCU_SUCCESS;
}

// back-projection half of iteration k (iter_backward over the parts)
static int slab_backward(dwcu_slab *sl, int k, bool next)
{
    const bool shb = (sl->s.method == DWCU_METHOD_SHB);
    TRY(slab_conv(sl, 1, shb, false));
    for (auto &pt : sl->parts) {
        dwcu_job *j = pt.j;
        if (!j) continue;
        CU(cudaSetDevice(pt.device));
        if (shb) {
            TRY(pass_x(j, XOP_UPDATE_SHB, next ? 1 : 0, j->S, j->xa, j->xb, j->xb, shb_alpha(k, sl->s.alphamax),
                       shb_alpha(k + 1, sl->s.alphamax)));
            std::swap(j->xa, j->xb);
        } else {
            TRY(pass_x(j, XOP_UPDATE_RL, next ? 1 : 0, j->S, j->xa, nullptr, j->xa, 0, 0));
        }
    }
    return DWCU_SUCCESS;
}

// every iteration (job_step_impl's schedule; launches stay eager)
static int slab_run(dwcu_slab *sl)
{
    PhaseRange pr("dwcu split iterations");
    if (!sl->setup_done) return fail(DWCU_ERROR_INVALID_VALUE, "run before setup");
    const bool shb = (sl->s.method == DWCU_METHOD_SHB);
    const bool fixed = (sl->s.iter_type == DWCU_ITER_FIXED);
    SlabPart &p0 = sl->lead();
    while (!sl->finished) {
        const int k = sl->k_next;
        if (fixed) {
            const bool last = (k == sl->it.niter - 1);
            if (!sl->spectrum_ready) TRY(slab_input(sl, k));
            TRY(slab_forward(sl, k, !(last && shb)));
            if (!(last && shb)) TRY(slab_backward(sl, k, !last));
            sl->spectrum_ready = !last;
            sl->done_iters = k + 1;
            sl->it.iter = k;
            sl->k_next = (k + 1 < sl->it.niter) ? k + 1 : -1;
            if (sl->k_next < 0) sl->finished = true;
            continue;
        }
        if (!sl->spectrum_ready) TRY(slab_input(sl, k));
        TRY(slab_forward(sl, k, true));
        float e = 0.f;
        CU(cudaSetDevice(p0.device));
        CU(cudaMemcpyAsync(&e, p0.j->err + k, sizeof(float), cudaMemcpyDeviceToHost, p0.stream));
        CU(cudaStreamSynchronize(p0.stream));
        sl->it.set(e);
        sl->done_iters = k + 1;
        if (sl->s.verbosity > 0) printf("Iteration %3d/%3d, %s=%.3e\n", k + 1, sl->it.niter,
                                        sl->s.metric == DWCU_METRIC_IDIV ? "Idiv" : "fMSE", e);
        const int kn = sl->it.next();
        if (kn >= 0) {
            TRY(slab_backward(sl, k, true));
            sl->spectrum_ready = true;
            sl->k_next = kn;
        } else {
            if (!shb) TRY(slab_backward(sl, k, false));  // RL returns x_{k+1}
            sl->spectrum_ready = false;
            sl->k_next = -1;
            sl->finished = true;
        }
    }
    return DWCU_SUCCESS;
}

// the result's image planes from every part into `out` (M x N x P, host)
static int slab_result(dwcu_slab *sl, float *out, dwcu_opts *so)
{
    PhaseRange pr("dwcu split result");
    const Geometry &g = sl->g;
    if (!sl->finished) return fail(DWCU_ERROR_NOT_READY, "the job has iterations left");
    const int n = (int) sl->parts.size();
    SlabPart &p0 = sl->lead();
    TRY(slab_join0(sl));
    CU(cudaSetDevice(p0.device));
    CU(cudaEventRecord(p0.j->ev2, p0.stream));
    int flags = 0;
    for (int p = 0; p < n; ++p) {
        SlabPart &pt = sl->parts[(size_t) p];
        if (!pt.j) continue;
        CU(cudaSetDevice(pt.device));
        for (long long l = 0; l < pt.pl; ++l) {
            const long long z = l * n + p;
            CU(cudaMemcpy2DAsync(out + z * g.M * g.N, sizeof(float) * g.M, pt.j->xa + l * g.Y * g.XP,
                                 sizeof(float) * g.XP, sizeof(float) * g.M, g.N, cudaMemcpyDeviceToHost, pt.stream));
        }
        JobScalars hs{};
        CU(cudaMemcpyAsync(&hs, pt.j->sc, sizeof hs, cudaMemcpyDeviceToHost, pt.stream));
        CU(cudaStreamSynchronize(pt.stream));
        flags |= hs.flags;
    }
    const int nerr = sl->done_iters;
    std::vector<float> errs((size_t) std::max(1, nerr));
    CU(cudaSetDevice(p0.device));
    if (nerr > 0) CU(cudaMemcpy(errs.data(), p0.j->err, sizeof(float) * nerr, cudaMemcpyDeviceToHost));
    if (flags & ~3) return fail(DWCU_ERROR_TIMEOUT, "a bounded wait in a pass gave up (flags 0x%x)", flags);
    if (so) {
        so->iterations_done = nerr;
        so->bg = sl->s.bg;
        so->work[0] = g.X; so->work[1] = g.Y; so->work[2] = g.Z;
        float ms_setup = 0, ms_loop = 0;
        cudaEventElapsedTime(&ms_setup, p0.j->ev0, p0.j->ev1);
        cudaEventElapsedTime(&ms_loop, p0.j->ev1, p0.j->ev2);
        so->seconds_setup = ms_setup * 1e-3;
        so->seconds_iterate = ms_loop * 1e-3;
        so->seconds_enqueue = 0;
        if (so->error_trace)
            for (int i = 0; i < nerr && i < so->trace_capacity; ++i) so->error_trace[i] = errs[(size_t) i];
        if (sl->s.verbosity > 0 && sl->s.iter_type == DWCU_ITER_FIXED)
            for (int i = 0; i < nerr; ++i)
                printf("Iteration %3d/%3d, %s=%.3e\n", i + 1, nerr,
                       sl->s.metric == DWCU_METRIC_IDIV ? "Idiv" : "fMSE", errs[(size_t) i]);
    }
    return DWCU_SUCCESS;
}

// one part of a job split over processes (one per GPU): this process's
// part on s->device; the other parts' spectra come from
// dwcu_slab_part_import
static int slab_create_part(long long M, long long N, long long P, long long pM, long long pN, long long pP,
                            const dwcu_opts *s, int nparts, int part, double *sync_buf, const dwcu_slab_sync *sync,
                            dwcu_slab **out)
{
    *out = nullptr;
    if (!s || !sync || !sync->barrier || !sync->allreduce || !sync_buf)
        return fail(DWCU_ERROR_INVALID_VALUE, "NULL argument");
    TRY(check_opts(*s));
    if (nparts < 1 || nparts > 64 || part < 0 || part >= nparts)
        return fail(DWCU_ERROR_INVALID_VALUE, "part %d of %d", part, nparts);
    Geometry g;
    TRY(make_geometry(M, N, P, pM, pN, pP, s->border_quality, g));
    if (g.wz)
        return fail(DWCU_ERROR_UNSUPPORTED, "job z size %lld needs periodic margins along z: not with parts", g.wP);
    if (nparts > g.Z) return fail(DWCU_ERROR_UNSUPPORTED, "%d parts for %lld z planes", nparts, g.Z);
    if (g.NKB * g.Y < nparts) return fail(DWCU_ERROR_UNSUPPORTED, "too few z-pass columns for %d parts", nparts);
    DeviceCtx *ctx = nullptr;
    TRY(get_ctx(s->device, &ctx));
    CU(cudaSetDevice(s->device));
    // every process must run the same plans: recorded choices (an imported
    // plan table) or the heuristic ones, never a measurement of its own
    tune_geometry(ctx, g, false);
    dwcu_slab *sl = new dwcu_slab();
    sl->s = *s;
    sl->g = g;
    sl->parts.resize((size_t) nparts);
    sl->local = part;
    sl->sync = *sync;
    sl->sync_buf = sync_buf;
    const char *tr = getenv("DWCU_SLAB_TRANSPOSE");
    sl->copies = tr && strcmp(tr, "copy") == 0;
    for (int p = 0; p < nparts; ++p) {
        SlabPart &o = sl->parts[(size_t) p];
        slab_layout(g.Z, g.P, g.NKB * g.Y * KB, nparts, p, &o.zl, &o.pl, &o.c0, &o.nc);
    }
    const int rc = slab_part_create(sl, part, s->device);
    if (rc != DWCU_SUCCESS) {
        slab_destroy(sl);
        return rc;
    }
    *out = sl;
    return DWCU_SUCCESS;
}

}  // namespace dwcu

extern "C" {

int dwcu_slab_part_create(int64_t M, int64_t N, int64_t P, int64_t pM, int64_t pN, int64_t pP, const dwcu_opts *s,
                          int32_t nparts, int32_t part, double *sync_buf, const dwcu_slab_sync *sync, dwcu_slab **out)
{
    if (!out) return fail(DWCU_ERROR_INVALID_VALUE, "out is NULL");
    return slab_create_part(M, N, P, pM, pN, pP, s, nparts, part, sync_buf, sync, out);
}

int dwcu_slab_part_export(dwcu_slab *sl, void *handle, int64_t *offset)
{
    if (!sl || !handle || !offset || sl->local < 0) return fail(DWCU_ERROR_INVALID_VALUE, "not a part of a split over processes");
    SlabPart &me = sl->lead();
    CU(cudaSetDevice(me.device));
    cudaIpcMemHandle_t h;
    CU(cudaIpcGetMemHandle(&h, me.j->base));
    memcpy(handle, &h, sizeof h);
    *offset = (int64_t) ((char *) me.j->S - me.j->base);
    return DWCU_SUCCESS;
}

int dwcu_slab_part_import(dwcu_slab *sl, int32_t part, const void *handle, int64_t offset)
{
    if (!sl || !handle || sl->local < 0) return fail(DWCU_ERROR_INVALID_VALUE, "not a part of a split over processes");
    if (part < 0 || part >= (int) sl->parts.size() || part == sl->local)
        return fail(DWCU_ERROR_INVALID_VALUE, "part %d: not another part of this split", part);
    SlabPart &o = sl->parts[(size_t) part];
    if (o.ipc_base) return fail(DWCU_ERROR_INVALID_VALUE, "part %d is mapped already", part);
    CU(cudaSetDevice(sl->lead().device));
    cudaIpcMemHandle_t h;
    memcpy(&h, handle, sizeof h);
    void *base = nullptr;
    CU(cudaIpcOpenMemHandle(&base, h, cudaIpcMemLazyEnablePeerAccess));
    o.ipc_base = base;
    o.S = reinterpret_cast<float2 *>((char *) base + offset);
    return DWCU_SUCCESS;
}

int dwcu_slab_part_run(dwcu_slab *sl, const float *im, const float *psf, float *out, dwcu_opts *so)
{
    if (!sl || !im || !psf || !out) return fail(DWCU_ERROR_INVALID_VALUE, "NULL argument");
    if (sl->local < 0) return fail(DWCU_ERROR_INVALID_VALUE, "not a part of a split over processes");
    if (sl->setup_done) return fail(DWCU_ERROR_INVALID_VALUE, "the part has run already");
    for (size_t q = 0; q < sl->parts.size(); ++q)
        if (!sl->parts[q].S)
            return fail(DWCU_ERROR_INVALID_VALUE, "part %zu's spectrum is not mapped (dwcu_slab_part_import)", q);
    if (so) so->iterations_done = 0;
    int rc = slab_setup(sl, im, psf);
    if (rc == DWCU_SUCCESS) rc = slab_run(sl);
    if (rc == DWCU_SUCCESS) rc = slab_result(sl, out, so);
    // no process frees or reuses its memory while another may still read it
    if (rc == DWCU_SUCCESS) rc = slab_sync_barrier(sl);
    if (rc == DWCU_SUCCESS) {
        CU(cudaSetDevice(sl->lead().device));
        CU(cudaStreamSynchronize(sl->lead().stream));
    }
    return rc;
}

void dwcu_slab_destroy(dwcu_slab *sl) { slab_destroy(sl); }

int dwcu_slab_layout(int64_t M, int64_t N, int64_t P, int64_t pM, int64_t pN, int64_t pP, int32_t border_quality,
                     int32_t nparts, int32_t part, int64_t *info)
{
    if (!info) return fail(DWCU_ERROR_INVALID_VALUE, "info is NULL");
    if (nparts < 1 || part < 0 || part >= nparts) return fail(DWCU_ERROR_INVALID_VALUE, "part %d of %d", part, nparts);
    Geometry g;
    TRY(make_geometry(M, N, P, pM, pN, pP, border_quality, g));
    long long zl, pl, c0, nc;
    const long long cols = g.NKB * g.Y * KB;
    slab_layout(g.Z, g.P, cols, nparts, part, &zl, &pl, &c0, &nc);
    info[0] = zl;
    info[1] = pl;
    info[2] = c0;
    info[3] = nc;
    info[4] = cols;
    info[5] = g.Z;
    return DWCU_SUCCESS;
}

int dwcu_deconvolve_slabs(const float *im, int64_t M, int64_t N, int64_t P, const float *psf, int64_t pM, int64_t pN,
                          int64_t pP, dwcu_opts *s, int32_t nparts, const int32_t *devices, float *out)
{
    if (!s || !im || !psf || !out) return fail(DWCU_ERROR_INVALID_VALUE, "NULL argument");
    s->iterations_done = 0;
    if (s->n_iter == 0) {
        // method_shb.c:101-105: nIter == 0 returns a copy of the image
        memcpy(out, im, sizeof(float) * (size_t) (M * N * P));
        return DWCU_SUCCESS;
    }
    int cur = 0;
    const bool had = cudaGetDevice(&cur) == cudaSuccess;
    dwcu_slab *sl = nullptr;
    int rc = slab_create(M, N, P, pM, pN, pP, s, nparts, devices, &sl);
    if (rc == DWCU_SUCCESS) rc = slab_setup(sl, im, psf);
    if (rc == DWCU_SUCCESS) rc = slab_run(sl);
    if (rc == DWCU_SUCCESS) rc = slab_result(sl, out, s);
    if (rc == DWCU_SUCCESS && s->bg_auto) s->bg = sl->s.bg;
    slab_destroy(sl);
    if (had) cudaSetDevice(cur);  // the caller's current device as it was
    return rc;
}

}  // extern "C"
