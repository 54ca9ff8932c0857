// Linear FFT convolution on the B200: pruned 3D R2C / C2R FFTs with the OTF
// product fused into the axial pass.
//
// Replaces deconlib's LinearFFTConvolver (deconvolution/linops_mlx.py:435-533)
// and FFTConvolver (:384-432).  With signal N = (Nz, Ny, Nx) zero-padded to
// the canvas F = (Fz, Fy, Fx), a convolution is five passes:
//
//   1. X R2C   N rows of x            -> S1[Nz][Ny][P]   (real FFT, length Fx)
//   2. Y FFT   S1, Ny non-zero points -> S2[Nz][Fy][P]
//   3. Z pass  S2 in place: FFT over Fz (Nz non-zero inputs), x OTF (or
//              conj(OTF) for the adjoint), inverse FFT, keep the first Nz
//   4. Y IFFT  S2 -> S1, keep the first Ny points
//   5. X C2R   S1 -> out, keep x < Nx, scale 1/(Fz Fy Fx), fused epilogue
//
// Zero padding never exists in memory (the loads return zeros) and only the
// Nz x Fy x (Fx/2+1) part of the spectrum that the crop can see is ever
// formed ("pruned" FFT).  P is the spectrum row pitch: Fx/2 + 1 rounded up to
// 16 complex values, so every 16-wide column tile of the strided passes
// reads whole 128-byte lines.
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include <algorithm>

#include "conv_impl.cuh"
#include "tma.cuh"
#include "colpipe.cuh"
#include "xpass.cuh"
#include "yzpass.cuh"

namespace dk {

// ---------------------------------------------------------------------------
// passes 2-4 on TMA: the same column transform with the tile moved by
// cp.async.bulk.tensor (one elected thread issues the boxes; an mbarrier with
// a bounded wait signals arrival; results leave through a TMA store).
// Power-of-two lengths L <= 512 with 16-column tiles (128-byte rows), so the
// shared-memory tile uses the TMA 128-byte swizzle layout (physw<1>).
// ---------------------------------------------------------------------------


template <int LS>
__global__ void __launch_bounds__(kFftThreads, (LS >= 512 ? 1 : 2)) k_colfft_tma(const __grid_constant__ ColTmaArgs a) {
    extern __shared__ unsigned char smraw[];
    float2* sm = reinterpret_cast<float2*>((reinterpret_cast<uintptr_t>(smraw) + 1023) & ~uintptr_t(1023));
    float2* so = sm + LS * 16;
    __shared__ uint64_t bar;
    const int tid = threadIdx.x;
    const int o = blockIdx.x / a.ntiles;
    const int c0 = (blockIdx.x - o * a.ntiles) * 32;  // float coordinate of the tile
    const bool otf = a.mode == COL_OTF || a.mode == COL_OTF_CONJ;
    const int nbox = (a.nin + a.src_box - 1) / a.src_box;
    if (tid == 0) {
        mbar_init(&bar, 1);
        fence_proxy_async_smem();
    }
    __syncthreads();
    if (tid == 0) {
        const uint32_t bytes = (uint32_t)(nbox * a.src_box * 128) + (otf ? (uint32_t)(LS * 128) : 0u);
        mbar_expect_tx(&bar, bytes);
        for (int i = 0; i < nbox; ++i) {
            const int r0 = i * a.src_box;
            if (a.src_jdim == 1) tma_load_3d(sm + r0 * 16, &a.src, c0, r0, o, &bar);
            else tma_load_3d(sm + r0 * 16, &a.src, c0, o, r0, &bar);
        }
        if (otf)
            for (int r0 = 0; r0 < LS; r0 += a.otf_box) tma_load_3d(so + r0 * 16, &a.otf, c0, o, r0, &bar);
    }
    // rows the boxes do not cover are the implicit zero padding
    for (int q = nbox * a.src_box * 16 + tid; q < LS * 16; q += blockDim.x) sm[q] = make_float2(0.f, 0.f);
    const bool ok = __syncthreads_and(mbar_wait_bounded(&bar, 0));
    if (!ok) return;
    const int t = tid & 15, jb = tid >> 4;
    if (a.mode == COL_INV) {
        fft_lines_static<LS, +1, 1, 1>(sm, 16, t, jb, a.tw, a.tws);
    } else {
        fft_lines_static<LS, -1, 1, 1>(sm, 16, t, jb, a.tw, a.tws);
    }
    if (otf) {
        for (int q = tid; q < LS * 16; q += blockDim.x) {
            const float2 w = so[q];
            sm[q] = a.mode == COL_OTF ? cmul(sm[q], w) : cmulc(sm[q], w);
        }
        __syncthreads();
        fft_lines_static<LS, +1, 1, 1>(sm, 16, t, jb, a.tw, a.tws);
    }
    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
        for (int r0 = 0; r0 < a.nout; r0 += a.dst_box) {
            if (a.dst_jdim == 1) tma_store_3d(&a.dst, c0, r0, o, sm + r0 * 16);
            else tma_store_3d(&a.dst, c0, o, r0, sm + r0 * 16);
        }
        tma_store_commit_and_wait();
    }
}

// ---------------------------------------------------------------------------
// host: axis planning and launches
// ---------------------------------------------------------------------------

bool plan_axis(int L, Axis& ax, int order) {
    ax = Axis{};
    ax.L = L;
    int n = L, e2 = 0;
    while (n % 2 == 0) {
        n /= 2;
        ++e2;
    }
    std::vector<int> r;
    int n8 = e2 / 3, rem = e2 % 3;
    if (rem == 1 && n8 > 0) {
        --n8;
        r.push_back(4);
        r.push_back(4);
    } else if (rem == 1) {
        r.push_back(2);
    } else if (rem == 2) {
        r.push_back(4);
    }
    for (int i = 0; i < n8; ++i) r.insert(r.begin(), 8);
    std::vector<int> odd;
    for (int p : {5, 3, 7}) {
        while (n % p == 0) {
            n /= p;
            odd.push_back(p);
        }
    }
    if (order == 1) r.insert(r.begin(), odd.begin(), odd.end());
    else r.insert(r.end(), odd.begin(), odd.end());
    if (n != 1 || (int)r.size() > kMaxStages) return false;
    ax.nst = (int)r.size();
    for (int i = 0; i < ax.nst; ++i) ax.rad |= (unsigned long long)r[i] << (4 * i);
    ax.tpl = static_length(L) ? (L + 31) / 32 : (L + kDynPPT - 1) / kDynPPT;
    return true;
}

static int threads_for(int T, const Axis& ax) {
    int n = T * ax.tpl;
    n = (int)round_up(n, 32);
    return std::max(n, 64);
}

// Kernel-class timing (decon_profile_start / _stop): CUDA events recorded
// on the launching stream around every launch of the selected classes.
struct ProfState {
    int mask = 0;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
    size_t used = 0;
};
static ProfState g_prof;

// Per (device, kernel, dynamic shared memory, block size): the occupancy is
// queried once; per (device, kernel) the shared-memory opt-in only ever rises
// to the largest size launched so far (a launch with less shared memory must
// not lower it under another plan's larger launches).  Later launches,
// including launches recorded into a CUDA graph, only look the entries up.
int kernel_prepare(void* fn, size_t smem, int nthr, int* per_sm) {
    static std::mutex mu;
    static std::map<std::tuple<int, void*, size_t, int>, int> done;
    static std::map<std::pair<int, void*>, size_t> opt_in;
    int dev = 0;
    DK_CUDA(cudaGetDevice(&dev));
    const auto key = std::make_tuple(dev, fn, smem, nthr);
    std::lock_guard<std::mutex> lock(mu);
    auto it = done.find(key);
    if (it != done.end()) {
        if (per_sm) *per_sm = it->second;
        return DECON_OK;
    }
    // the 48 KB default covers static plus dynamic shared memory: opt in
    // whenever their sum exceeds it
    cudaFuncAttributes fa{};
    DK_CUDA(cudaFuncGetAttributes(&fa, fn));
    if (smem + fa.sharedSizeBytes > 48 * 1024) {
        size_t& cur = opt_in[std::make_pair(dev, fn)];
        if (smem > cur) {
            DK_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            cur = smem;
        }
    }
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, nthr, smem) != cudaSuccess) {
        cudaGetLastError();
        occ = 0;
    }
    done[key] = occ;
    if (per_sm) *per_sm = occ;
    return DECON_OK;
}

static int launch(void* fn, int64_t nblk, int nthr, size_t smem, cudaStream_t st, void* args,
                  int cls) {
    DK_TRY(kernel_prepare(fn, smem, nthr, nullptr));
    if (nblk <= 0) return DECON_OK;
    if (nblk > 0x7fffffffLL) return fail(DECON_ERR_UNSUPPORTED, "grid too large");
    void* params[] = {args};
    const bool prof = (g_prof.mask & cls) != 0;
    if (prof) {
        if (g_prof.used == g_prof.ev.size()) {
            cudaEvent_t a, b;
            DK_CUDA(cudaEventCreate(&a));
            DK_CUDA(cudaEventCreate(&b));
            g_prof.ev.emplace_back(a, b);
        }
        DK_CUDA(cudaEventRecord(g_prof.ev[g_prof.used].first, st));
    }
    DK_CUDA(cudaLaunchKernel(fn, dim3((unsigned)nblk), dim3(nthr), params, smem, st));
    count_launch();
    if (prof) {
        DK_CUDA(cudaEventRecord(g_prof.ev[g_prof.used].second, st));
        ++g_prof.used;
    }
    return DECON_OK;
}

}  // namespace dk

extern "C" int decon_device_status(void* stream) {
    using namespace dk;
    DK_CUDA(cudaStreamSynchronize(as_stream(stream)));
    int flag = 0;
    DK_CUDA(cudaMemcpyFromSymbol(&flag, g_wait_timeout, sizeof(int)));
    if (flag) return fail(DECON_ERR_TIMEOUT, "a bounded TMA wait gave up; results are invalid");
    return DECON_OK;
}

extern "C" int decon_device_status_clear(void* stream) {
    using namespace dk;
    DK_CUDA(cudaStreamSynchronize(as_stream(stream)));
    const int zero = 0;
    DK_CUDA(cudaMemcpyToSymbol(g_wait_timeout, &zero, sizeof(int)));
    return DECON_OK;
}

namespace dk {

// One CTA waits, through the kernels' own bounded wait, on an mbarrier that
// no thread arrives at and no copy completes: every poll fails, the wait
// gives up after `polls` polls, raises g_wait_timeout and the CTA returns.
// Nothing is in flight and nothing is written but the flag.
__global__ void k_wait_probe(unsigned polls) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_proxy_async_smem();
    }
    __syncthreads();
    if (threadIdx.x == 0) (void)mbar_wait_bounded(&bar, 0, polls);
}

}  // namespace dk

extern "C" int decon_test_wait_timeout(unsigned polls, void* stream) {
    using namespace dk;
    if (polls == 0 || polls > (1u << 16))
        return fail(DECON_ERR_VALUE, "decon_test_wait_timeout: polls must be in [1, 65536]");
    k_wait_probe<<<1, 32, 0, as_stream(stream)>>>(polls);
    DK_LAUNCHED();
    return DECON_OK;
}

extern "C" int decon_profile_start(int class_mask) {
    dk::g_prof.mask = class_mask;
    dk::g_prof.used = 0;
    return DECON_OK;
}

extern "C" int decon_profile_stop(double* ms_total, int64_t* launches) {
    using namespace dk;
    double tot = 0.0;
    for (size_t i = 0; i < g_prof.used; ++i) {
        DK_CUDA(cudaEventSynchronize(g_prof.ev[i].second));
        float ms = 0.f;
        DK_CUDA(cudaEventElapsedTime(&ms, g_prof.ev[i].first, g_prof.ev[i].second));
        tot += ms;
    }
    if (ms_total) *ms_total = tot;
    if (launches) *launches = (int64_t)g_prof.used;
    g_prof.mask = 0;
    g_prof.used = 0;
    return DECON_OK;
}

namespace dk {

int launch_xr2c(const ConvPlan& p, int pro, const float* in, Win3 win, float cval, float bg,
                int64_t nz_rows, float2* out, cudaStream_t st, int64_t kstride) {
    XR2CArgs a{};
    a.kstride = kstride;
    a.in = in;
    a.cval = cval;
    a.bg = bg;
    a.Nz = nz_rows;
    a.Ny = pro == PRO_KERNEL ? p.F[1] : p.N[1];
    a.Nx = pro == PRO_KERNEL ? p.F[2] : p.N[2];
    a.win = win;
    a.Kz = p.K[0];
    a.Ky = p.K[1];
    a.Kx = p.K[2];
    a.pz = (p.K[0] + 1) / 2;
    a.py = (p.K[1] + 1) / 2;
    a.px = (p.K[2] + 1) / 2;
    a.kdiv = p.kdiv;
    a.out = out;
    a.P = p.P;
    a.Hx = (int)p.Hx;
    a.odd = p.odd;
    a.ax = p.ax_x;
    a.twx = p.twx;
    a.vec4 = pro == PRO_ARRAY && in != nullptr && !p.odd && (a.Nx % 4) == 0 && win.oz == 0 &&
             win.oy == 0 && win.ox == 0 && win.wz == p.N[0] && win.wy == p.N[1] &&
             win.wx == p.N[2] && (reinterpret_cast<uintptr_t>(in) & 15) == 0;
    // the 2x adjoint prologue reads coarse rows of Nx / 2 floats as float4
    const bool up2_vec = pro == PRO_UP2 && (a.Nx % 8) == 0 && (reinterpret_cast<uintptr_t>(in) & 15) == 0;
    if (pro == PRO_UP2) a.vec4 = up2_vec;
    a.T = p.T_x;
    a.nrows = nz_rows * a.Ny;
    if (static_length(a.ax.L))
        if (a.T != x_lines(a.ax.L)) return fail(DECON_ERR_UNSUPPORTED, "X pass lines per CTA mismatch");
    {
        const int L = a.ax.L;
        const int64_t nin = p.odd ? std::min<int64_t>(a.Nx, L) : std::min<int64_t>((a.Nx + 1) / 2, L);
        a.fd_q4 = make_fastdiv(std::max<int64_t>(1, pro == PRO_UP2 ? a.Nx / 8 : a.Nx / 4));
        a.fd_H = make_fastdiv(a.Hx);
        a.fd_nin = make_fastdiv(std::max<int64_t>(1, nin));
        a.fd_np = make_fastdiv(L / 2 + 1);
    }
    const int nthr = threads_for(a.T, a.ax);
    const int64_t nblk = cdiv(a.nrows, a.T);
    const size_t smem = (size_t)a.T * a.ax.L * sizeof(float2);
    void* fn = pick_xr2c_kernel(pro, a.ax.L);
    if (!fn) return fail(DECON_ERR_VALUE, "bad prologue %d", pro);
    return launch(fn, nblk, nthr, smem, st, &a, PROF_XR2C);
}

int launch_col(const ConvPlan& p, const Axis& ax, int T, int mode, const float2* src,
               int64_t src_os, int64_t src_js, int nin, float2* dst, int64_t dst_os,
               int64_t dst_js, int nout, int64_t nouter, cudaStream_t st) {
    ColArgs a{};
    a.src = src;
    a.dst = dst;
    a.src_os = src_os;
    a.src_js = src_js;
    a.dst_os = dst_os;
    a.dst_js = dst_js;
    a.nin = nin;
    a.nout = nout;
    a.ncols = (int)p.Hx;
    a.T = T;
    a.ax = ax;
    a.mode = mode;
    a.otf = p.otf;
    a.otf_js = p.F[1] * p.P;
    a.otf_os = p.P;
    a.ntiles = (int)cdiv(p.Hx, T);
    const int nthr = threads_for(T, ax);
    const int64_t nblk = nouter * a.ntiles;
    const size_t smem = (size_t)T * ax.L * sizeof(float2);
    return launch(pick_colfft_kernel(ax.L), nblk, nthr, smem, st, &a,
                  (mode == COL_OTF || mode == COL_OTF_CONJ) ? PROF_ZOTF : PROF_COL);
}

int launch_xc2r(const ConvPlan& p, int epi, const float2* in, Win3 win, float* out,
                const float* aux0, const float* aux1, float bg, double* partials, int* nblk_out,
                cudaStream_t st) {
    XC2RArgs a{};
    a.in = in;
    a.P = p.P;
    a.Ny = p.N[1];
    a.Nx = p.N[2];
    a.nrows = p.N[0] * p.N[1];
    a.Hx = (int)p.Hx;
    a.odd = p.odd;
    a.ax = p.ax_x;
    a.twx = p.twx;
    {
        const bool full = win.oz == 0 && win.oy == 0 && win.ox == 0 && win.wz == p.N[0] &&
                          win.wy == p.N[1] && win.wx == p.N[2];
        auto al = [](const void* q) { return q == nullptr || (reinterpret_cast<uintptr_t>(q) & 15) == 0; };
        a.vec4 = full && !p.odd && (p.N[2] % 4) == 0 && al(out) && al(aux0) && al(aux1);
    }
    a.T = p.T_x;
    if (static_length(a.ax.L))
        if (a.T != x_lines(a.ax.L)) return fail(DECON_ERR_UNSUPPORTED, "X pass lines per CTA mismatch");
    a.scale = (float)(1.0 / ((double)p.F[0] * (double)p.F[1] * (double)p.F[2]));
    a.win = win;
    a.out = out;
    a.aux0 = aux0;
    a.aux1 = aux1;
    a.bg = bg;
    a.partials = partials;
    a.kstride = use_yz(p) ? p.N[0] * p.N[1] : 0;
    {
        const int L = a.ax.L;
        a.fd_L = make_fastdiv(L);
        a.fd_h2 = make_fastdiv(std::max(1, L / 2));
        a.fd_npair = make_fastdiv(L / 2 + 1);
        a.fd_q4 = make_fastdiv(std::max<int64_t>(1, epi == EPI_DOWN2 ? a.Nx / 2 : a.Nx / 4));
        a.fd_Nx = make_fastdiv(a.Nx);
    }
    if (epi == EPI_DOWN2) {
        // whole 2 x 2 x 2 blocks per CTA: T / 2 lines from each of two planes
        a.vec4 = 0;
        if (p.odd || (p.N[0] | p.N[1] | p.N[2]) & 1 || a.T < 4 || p.N[1] % (a.T / 2) != 0)
            return fail(DECON_ERR_UNSUPPORTED, "2x area-sum epilogue: extents must be even and Ny a "
                                               "multiple of %d", a.T / 2);
    }
    const int nthr = threads_for(a.T, a.ax);
    const int64_t nblk = cdiv(a.nrows, a.T);
    if (nblk_out) *nblk_out = (int)nblk;
    const size_t smem = (size_t)a.T * a.ax.L * sizeof(float2);
    void* fn = pick_xc2r_kernel(epi, a.ax.L);
    if (!fn) return fail(DECON_ERR_VALUE, "bad epilogue %d", epi);
    return launch(fn, nblk, nthr, smem, st, &a, PROF_XC2R);
}

static void* pick_col_tma(int L) {
    switch (L) {
        case 64: return (void*)k_colfft_tma<64>;
        case 128: return (void*)k_colfft_tma<128>;
        case 256: return (void*)k_colfft_tma<256>;
        case 512: return (void*)k_colfft_tma<512>;
        case 80: return (void*)k_colfft_tma<80>;
        case 96: return (void*)k_colfft_tma<96>;
        case 160: return (void*)k_colfft_tma<160>;
        case 192: return (void*)k_colfft_tma<192>;
        case 240: return (void*)k_colfft_tma<240>;
        default: return nullptr;
    }
}

// Lengths with a TMA column kernel: the powers of two up to 512, and the
// other compile-time lengths up to 256 (one TMA box spans the whole line, so
// no box reaches past the tile).
bool tma_length_ok(int L) {
    return L == 64 || L == 128 || L == 256 || L == 512 || L == 80 || L == 96 || L == 160 || L == 192 ||
           L == 240;
}

static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 enc = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            enc = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
        else
            cudaGetLastError();
    }
    return enc;
}

bool encode_half_plane_map(CUtensorMap* map, const __half2* base, int64_t pitch, int64_t d1, int64_t d2,
                           int b2) {
    const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return false;
    // one half2 = one 4-byte element; rows of 16 elements (64 bytes), no swizzle
    cuuint64_t dims[3] = {(cuuint64_t)pitch, (cuuint64_t)d1, (cuuint64_t)d2};
    cuuint64_t strides[2] = {(cuuint64_t)(pitch * sizeof(__half2)),
                             (cuuint64_t)(pitch * sizeof(__half2) * d1)};
    cuuint32_t box[3] = {16u, 1u, (cuuint32_t)b2};
    cuuint32_t estr[3] = {1u, 1u, 1u};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<__half2*>(base), dims, strides,
                     box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

bool encode_spectrum_map(CUtensorMap* map, const float2* base, int64_t pitch, int64_t d1, int64_t d2,
                         int b1, int b2) {
    const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return false;
    cuuint64_t dims[3] = {(cuuint64_t)(2 * pitch), (cuuint64_t)d1, (cuuint64_t)d2};
    cuuint64_t strides[2] = {(cuuint64_t)(2 * pitch * sizeof(float)),
                             (cuuint64_t)(2 * pitch * sizeof(float) * d1)};
    cuuint32_t box[3] = {32u, (cuuint32_t)b1, (cuuint32_t)b2};
    cuuint32_t estr[3] = {1u, 1u, 1u};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float2*>(base), dims, strides,
                     box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// One column pass on TMA.  src/dst/otf maps come from the plan.
// Pipelined kernel for (L, mode, nin, nout), or nullptr.  R x R (SPLIT 1) for
// L = 64, 256; the half-zero split (SPLIT 2) for L = 128, 512 when the
// non-zero input / kept output fits in half the axis.
// h16: the axial (OTF) modes read the FP16 OTF (mixed precision).
static void* pick_pipe(int L, int mode, int nin, int nout, int* R, int* split, bool h16 = false,
                       bool lean = false) {
    const bool otf = mode == COL_OTF || mode == COL_OTF_CONJ;
    const bool half_ok = (mode == COL_FWD && nin <= L / 2) || (mode == COL_INV && nout <= L / 2) ||
                         (otf && nin <= L / 2 && nout <= L / 2);
#define DK_PIPE(RR, SS)                                                                          \
    do {                                                                                         \
        *R = RR;                                                                                 \
        *split = SS;                                                                             \
        switch (mode) {                                                                          \
            case COL_FWD: return (void*)k_col_pipe<RR, SS, COL_FWD>;                             \
            case COL_INV: return (void*)k_col_pipe<RR, SS, COL_INV>;                             \
            case COL_OTF:                                                                        \
                return h16 ? (lean ? (void*)k_col_pipe<RR, SS, COL_OTF, true, true>              \
                                   : (void*)k_col_pipe<RR, SS, COL_OTF, true>)                  \
                           : (lean ? (void*)k_col_pipe<RR, SS, COL_OTF, false, true>            \
                                   : (void*)k_col_pipe<RR, SS, COL_OTF>);                       \
            case COL_OTF_CONJ:                                                                   \
                return h16 ? (lean ? (void*)k_col_pipe<RR, SS, COL_OTF_CONJ, true, true>         \
                                   : (void*)k_col_pipe<RR, SS, COL_OTF_CONJ, true>)             \
                           : (lean ? (void*)k_col_pipe<RR, SS, COL_OTF_CONJ, false, true>       \
                                   : (void*)k_col_pipe<RR, SS, COL_OTF_CONJ>);                  \
        }                                                                                        \
    } while (0)
    if (L == 256) DK_PIPE(16, 1);
    if (L == 64) DK_PIPE(8, 1);
    if (L == 128 && half_ok) DK_PIPE(8, 2);
#undef DK_PIPE
    if (L == 512 && half_ok && !otf) {
        *R = 16;
        *split = 2;
        return mode == COL_FWD ? (void*)k_col_pipe<16, 2, COL_FWD> : (void*)k_col_pipe<16, 2, COL_INV>;
    }
    return nullptr;
}

static bool launch_col_pipe(const ConvPlan& p, const Axis& ax, int mode, const CUtensorMap& src,
                            int src_jdim, int src_box, int nin, const CUtensorMap& dst, int dst_jdim,
                            int dst_box, int nout, int64_t nouter, cudaStream_t st, int* status) {
    int R = 0, split = 0;
    const bool otf_mode = mode == COL_OTF || mode == COL_OTF_CONJ;
    const bool h16 = otf_mode && p.precision == 1 && p.otf16 != nullptr;
    // axial pass of length 256: the lean two-CTA kernel (measured 153 vs 166 us
    // at 128x256x256 on the B200); DECON_PIPE_LEAN=0 / 1 overrides.  Its FP16
    // form stages the half OTF tile by TMA (needs the plan's half-OTF map).
    const char* le = getenv("DECON_PIPE_LEAN");
    const bool lean = otf_mode && (!h16 || p.tma_otf16) &&
                      (le ? le[0] == '1' : (ax.L == 256 && !(p.sched & DECON_SCHED_LEAN_OFF)));
    const bool no_pipe = getenv("DECON_NO_PIPE") || (p.sched & DECON_SCHED_NO_PIPE);
    void* fn = no_pipe ? nullptr : pick_pipe(ax.L, mode, nin, nout, &R, &split, h16, lean);
    if (!fn) return false;
    PipeArgs a;
    memset(&a, 0, sizeof(a));
    a.src = src;
    a.dst = dst;
    a.otf = p.otf;
    a.otf16 = p.otf16;
    a.otf_inv = p.otf_inv;
    a.otfmap = p.tm_otf_z;
    a.otfmap16 = p.tm_otf16_z;
    a.otf_box = p.otf_box;
    a.otf_js = p.F[1] * p.P;
    a.otf_os = p.P;
    a.tw = ax.tw;
    a.tws = ax.tws;
    a.nin = nin;
    a.nout = nout;
    a.ntiles = (int)cdiv(p.Hx, 16);
    a.nouter = (int)nouter;
    a.src_jdim = src_jdim;
    a.dst_jdim = dst_jdim;
    a.src_box = src_box;
    a.dst_box = dst_box;
    const int L = ax.L;
    const int ns = pipe_slots(L, lean);
    // OTF tile: FP32 in each ring slot, or (lean) one buffer of FP32 or FP16
    const bool otf_tile = otf_mode && !h16;
    const size_t tile_bytes = (size_t)L * 16 * sizeof(float2);
    const size_t smem = 1024 + (size_t)ns * tile_bytes * (otf_tile && !lean ? 2 : 1) +
                        (otf_mode && lean ? (h16 ? tile_bytes / 2 : tile_bytes) : 0);
    const int nthr = 16 * R;
    *status = DECON_OK;
    int per_sm = 1;
    if ((*status = kernel_prepare(fn, smem, nthr, &per_sm)) != DECON_OK) return true;
    if (per_sm < 1) per_sm = 1;
    const int64_t total = nouter * a.ntiles;
    const int64_t grid = std::min<int64_t>(total, (int64_t)sm_count() * per_sm);
    *status = launch(fn, grid, nthr, smem, st, &a,
                     (mode == COL_OTF || mode == COL_OTF_CONJ) ? PROF_ZOTF : PROF_COL);
    return true;
}

bool zpass_pipelined(const ConvPlan& p) {
    if (!p.tma_z || getenv("DECON_NO_PIPE") || (p.sched & (DECON_SCHED_NO_PIPE | DECON_SCHED_NO_TMA)))
        return false;
    int R = 0, split = 0;
    return pick_pipe(p.ax_z.L, COL_OTF, (int)p.N[0], (int)p.N[0], &R, &split) != nullptr;
}

static int launch_col_tma(const ConvPlan& p, const Axis& ax, int mode, const CUtensorMap& src,
                          int src_jdim, int src_box, int nin, const CUtensorMap& dst, int dst_jdim,
                          int dst_box, int nout, int64_t nouter, cudaStream_t st) {
    int pst = DECON_OK;
    if (launch_col_pipe(p, ax, mode, src, src_jdim, src_box, nin, dst, dst_jdim, dst_box, nout,
                        nouter, st, &pst))
        return pst;
    ColTmaArgs a;
    memset(&a, 0, sizeof(a));
    a.src = src;
    a.dst = dst;
    if (mode == COL_OTF || mode == COL_OTF_CONJ) a.otf = p.tm_otf_z;
    a.nin = nin;
    a.nout = nout;
    a.ntiles = (int)cdiv(p.Hx, 16);
    a.mode = mode;
    a.src_jdim = src_jdim;
    a.dst_jdim = dst_jdim;
    a.src_box = src_box;
    a.dst_box = dst_box;
    a.otf_box = p.otf_box;
    a.tw = ax.tw;
    a.tws = ax.tws;
    const int L = ax.L;
    const int nthr = std::max(64, 16 * ((L + 31) / 32));  // 16 lines x the static path's threads per line
    const bool otf = mode == COL_OTF || mode == COL_OTF_CONJ;
    const size_t smem = 1024 + (size_t)L * 16 * sizeof(float2) * (otf ? 2 : 1);
    return launch(pick_col_tma(L), nouter * a.ntiles, nthr, smem, st, &a,
                  otf ? PROF_ZOTF : PROF_COL);
}

// ---------------------------------------------------------------------------
// fused Y / axial pass (yzpass.cuh)
// ---------------------------------------------------------------------------

bool yz_supported(const int64_t N[3], const int64_t F[3]) {
    const bool fy = F[1] == 256 || F[1] == 512, fz = F[0] == 128 || F[0] == 256;
    return fy && fz && N[1] <= F[1] / 2 && N[0] <= F[0] / 2 && N[1] % 2 == 0 && N[0] >= 1 &&
           N[1] >= 2;
}

bool use_yz(const ConvPlan& p) {
    // opt-in: the plan's schedule asks for it, or DECON_YZ=1 for every plan
    // (on the B200 the fused pass measured slower than the separate passes:
    // it is instruction-bound, 15 eight-CTA clusters occupy 120 of 148 SMs)
    const bool want = (p.sched & DECON_SCHED_FUSED) || getenv("DECON_YZ") != nullptr;
    return want && p.otft != nullptr && p.precision == 0 && getenv("DECON_NO_YZ") == nullptr;
}

// out[(kx * Fy + ky) * Fz + kz] = otf[(kz * Fy + ky) * P + kx]: 32 x 32 tiles
// of (kz, kx) per ky through shared memory.
__global__ void k_otf_kmajor(const float2* __restrict__ otf, int Fz, int Fy, int64_t P, int Hx,
                             float2* __restrict__ out) {
    __shared__ float2 t[32][33];
    const int ky = blockIdx.z;
    const int kx0 = blockIdx.x * 32, kz0 = blockIdx.y * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int kz = kz0 + i, kx = kx0 + threadIdx.x;
        if (kz < Fz && kx < Hx) t[i][threadIdx.x] = otf[((int64_t)kz * Fy + ky) * P + kx];
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int kx = kx0 + i, kz = kz0 + threadIdx.x;
        if (kz < Fz && kx < Hx) out[((int64_t)kx * Fy + ky) * Fz + kz] = t[threadIdx.x][i];
    }
}

int build_otf_kmajor(const ConvPlan& p, cudaStream_t st) {
    if (!p.otft) return DECON_OK;
    const dim3 grid((unsigned)cdiv(p.Hx, 32), (unsigned)cdiv(p.F[0], 32), (unsigned)p.F[1]);
    k_otf_kmajor<<<grid, dim3(32, 8), 0, st>>>(p.otf, (int)p.F[0], (int)p.F[1], p.P, (int)p.Hx, p.otft);
    DK_LAUNCHED();
    return DECON_OK;
}

template <int FY, int FZ, int C, int NT>
static void* pick_yz_fz(bool adjoint) {
    return adjoint ? (void*)k_yz<FY, FZ, COL_OTF_CONJ, C, NT> : (void*)k_yz<FY, FZ, COL_OTF, C, NT>;
}

template <int C, int NT>
static void* pick_yz_c(int64_t Fy, int64_t Fz, bool adjoint) {
    if (Fy == 512 && Fz == 256) return pick_yz_fz<512, 256, C, NT>(adjoint);
    if (Fy == 512 && Fz == 128) return pick_yz_fz<512, 128, C, NT>(adjoint);
    if (Fy == 256 && Fz == 256) return pick_yz_fz<256, 256, C, NT>(adjoint);
    if (Fy == 256 && Fz == 128) return pick_yz_fz<256, 128, C, NT>(adjoint);
    return nullptr;
}

// Cluster shape of the fused pass: 8 x 512 threads (default) or, with
// DECON_YZ_CLUSTER=16, 16 x 256 threads (two CTAs per SM).
static int yz_cluster_size() {
    const char* e = getenv("DECON_YZ_CLUSTER");
    return (e && atoi(e) == 16) ? 16 : 8;
}

static void* pick_yz(int64_t Fy, int64_t Fz, bool adjoint, int C) {
    return C == 16 ? pick_yz_c<16, 256>(Fy, Fz, adjoint) : pick_yz_c<8, 512>(Fy, Fz, adjoint);
}

// Clusters of k_yz resident at once on this device (cached per kernel).
static int yz_clusters(void* fn, size_t smem, int C, int NT) {
    static std::mutex mu;
    static std::map<std::pair<int, void*>, int> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    auto key = std::make_pair(dev, fn);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C * 64);
    cfg.blockDim = dim3(NT);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, fn, &cfg) != cudaSuccess || n < 1) {
        cudaGetLastError();
        n = std::max(1, sm_count() / C);
    }
    cache[key] = n;
    return n;
}

static int launch_yz(const ConvPlan& p, bool adjoint, cudaStream_t st) {
    const int C = yz_cluster_size(), NT = C == 16 ? 256 : 512;
    void* fn = pick_yz(p.F[1], p.F[0], adjoint, C);
    if (!fn) return fail(DECON_ERR_UNSUPPORTED, "fused Y / axial pass: unsupported canvas");
    YZArgs a;
    a.s1t = p.s1;
    a.otft = p.otft;
    a.twy = p.twy;
    a.twz = p.twz;
    a.Nz = (int)p.N[0];
    a.Ny = (int)p.N[1];
    a.Hx = (int)p.Hx;
    const size_t smem = yz_smem_bytes((int)p.F[1], (int)p.F[0], C);
    if (C > 8) {
        static std::mutex mu;
        static std::map<std::pair<int, void*>, bool> done;
        int dev = 0;
        cudaGetDevice(&dev);
        std::lock_guard<std::mutex> lock(mu);
        if (!done[std::make_pair(dev, fn)]) {
            DK_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
            done[std::make_pair(dev, fn)] = true;
        }
    }
    DK_TRY(kernel_prepare(fn, smem, NT, nullptr));
    const int ncl = (int)std::min<int64_t>(p.Hx, yz_clusters(fn, smem, C, NT));
    // a cluster launch, timed like the other passes when profiling is on
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(ncl * C));
    cfg.blockDim = dim3(NT);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    void* params[] = {&a};
    const bool prof = (g_prof.mask & PROF_ZOTF) != 0;
    if (prof) {
        if (g_prof.used == g_prof.ev.size()) {
            cudaEvent_t e0, e1;
            DK_CUDA(cudaEventCreate(&e0));
            DK_CUDA(cudaEventCreate(&e1));
            g_prof.ev.emplace_back(e0, e1);
        }
        DK_CUDA(cudaEventRecord(g_prof.ev[g_prof.used].first, st));
    }
    DK_CUDA(cudaLaunchKernelExC(&cfg, fn, params));
    count_launch();
    if (prof) {
        DK_CUDA(cudaEventRecord(g_prof.ev[g_prof.used].second, st));
        ++g_prof.used;
    }
    return DECON_OK;
}

// Forward spectrum: x (window in N-space) -> S2 (after the Y pass), or, with
// the fused Y / axial pass, -> the kx-major S1 (X pass only).
int spectrum_forward(const ConvPlan& p, int pro, const float* in, Win3 win, float cval, float bg,
                     cudaStream_t st) {
    const int64_t Nz = p.N[0], Ny = p.N[1], Fy = p.F[1], P = p.P;
    if (use_yz(p)) return launch_xr2c(p, pro, in, win, cval, bg, Nz, p.s1, st, Nz * Ny);
    DK_TRY(launch_xr2c(p, pro, in, win, cval, bg, Nz, p.s1, st));
    if (p.tma_y && !(p.sched & DECON_SCHED_NO_TMA)) {
        DK_TRY(launch_col_tma(p, p.ax_y, COL_FWD, p.tm_s1_j1, 1, p.s1_box, (int)Ny, p.tm_s2_j1, 1,
                              p.s2y_box, (int)Fy, Nz, st));
    } else {
        DK_TRY(launch_col(p, p.ax_y, p.T_y, COL_FWD, p.s1, Ny * P, P, (int)Ny, p.s2, Fy * P, P,
                          (int)Fy, Nz, st));
    }
    return DECON_OK;
}

// Z pass (x OTF or conj OTF) and the inverse Y pass: S2 -> S1.
int spectrum_filter_back(const ConvPlan& p, bool adjoint, cudaStream_t st) {
    if (use_yz(p)) return launch_yz(p, adjoint, st);
    const int64_t Nz = p.N[0], Ny = p.N[1], Fy = p.F[1], P = p.P;
    const int mode = adjoint ? COL_OTF_CONJ : COL_OTF;
    const bool tma = !(p.sched & DECON_SCHED_NO_TMA);
    if (p.tma_z && tma) {
        DK_TRY(launch_col_tma(p, p.ax_z, mode, p.tm_s2_j2, 2, p.s2z_box, (int)Nz, p.tm_s2_j2, 2,
                              p.s2z_box, (int)Nz, Fy, st));
    } else {
        DK_TRY(launch_col(p, p.ax_z, p.T_z, mode, p.s2, P, Fy * P, (int)Nz, p.s2, P, Fy * P,
                          (int)Nz, Fy, st));
    }
    if (p.tma_y && tma) {
        DK_TRY(launch_col_tma(p, p.ax_y, COL_INV, p.tm_s2_j1, 1, p.s2y_box, (int)Fy, p.tm_s1_j1, 1,
                              p.s1_box, (int)Ny, Nz, st));
    } else {
        DK_TRY(launch_col(p, p.ax_y, p.T_y, COL_INV, p.s2, Fy * P, P, (int)Fy, p.s1, Ny * P, P,
                          (int)Ny, Nz, st));
    }
    return DECON_OK;
}

}  // namespace dk
