// C ABI: error state, FFT sizing, convolution plans and the fused
// Richardson-Lucy entry points (include/decon_b200.h).
#include <atomic>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include <map>
#include "conv_impl.cuh"

namespace dk {

static thread_local std::string g_err;
static std::atomic<long long> g_launches{0};

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void count_launches(int64_t n) { g_launches.fetch_add((long long)n, std::memory_order_relaxed); }

void set_error(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
}

int fail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

static cudaStream_t setup_stream() {
    static std::mutex mu;
    static std::map<int, cudaStream_t> streams;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    auto it = streams.find(dev);
    if (it != streams.end()) return it->second;
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    streams[dev] = s;
    return s;
}

int upload_blocking(void* dst, const void* src, size_t bytes) {
    const cudaStream_t s = setup_stream();
    if (!s) return fail(DECON_ERR_CUDA, "set-up stream creation failed");
    DK_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
    DK_CUDA(cudaStreamSynchronize(s));
    return DECON_OK;
}

int memset_blocking(void* dst, int value, size_t bytes) {
    const cudaStream_t s = setup_stream();
    if (!s) return fail(DECON_ERR_CUDA, "set-up stream creation failed");
    DK_CUDA(cudaMemsetAsync(dst, value, bytes, s));
    DK_CUDA(cudaStreamSynchronize(s));
    return DECON_OK;
}

int sm_count() {
    static int cached[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (!cached[dev]) {
        int n = 0;
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        cached[dev] = n > 0 ? n : 148;
    }
    return cached[dev];
}

int max_abs2(const float2* z, int64_t rows, int64_t cols, int64_t pitch, double* out,
             double* partials, cudaStream_t st);

// Twiddle table W_L^m = exp(-2 pi i m / L), m < L, computed in double.
static int make_twiddles(int L, float2** out) {
    std::vector<float2> h(std::max(L, 1));
    for (int m = 0; m < L; ++m) {
        const double a = -2.0 * M_PI * (double)m / (double)L;
        h[m] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    DK_CUDA(cudaMalloc(out, h.size() * sizeof(float2)));
    DK_TRY(upload_blocking(*out, h.data(), h.size() * sizeof(float2)));
    return DECON_OK;
}

static void free_plan(ConvPlan* p) {
    if (!p) return;
    cudaFree(p->otft);
    cudaFree(p->otf16);
    cudaFree(p->otf_inv);
    cudaFree(p->otf);
    cudaFree(p->s1);
    cudaFree(p->s2);
    cudaFree(p->twx);
    cudaFree(p->twy);
    cudaFree(p->twz);
    cudaFree(p->dscal);
    cudaFree(p->partials);
}

static int dev_alloc(void** p, size_t bytes, const char* what) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(e == cudaErrorMemoryAllocation ? DECON_ERR_OOM : DECON_ERR_CUDA,
                    "cudaMalloc of %zu bytes for %s failed: %s", bytes, what, cudaGetErrorString(e));
    }
    return DECON_OK;
}

// Elementwise helpers used by the RL set-up.
__global__ void k_rl_mask(float* __restrict__ x, float* __restrict__ sens, const double* smax,
                          int64_t n, int clamp_init) {
    // rl_mlx.py:130-133  floor = max(max(sens) * 1e-6, 1e-10); active = sens > floor
    const float fl = fmaxf((float)(*smax) * 1e-6f, 1e-10f);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float s = sens[i];
        const bool act = s > fl;
        sens[i] = act ? s : 0.f;
        const float xv = fmaxf(x[i], 1e-6f);  // rl_mlx.py:125,127 max(., 1e-6)
        x[i] = act ? xv : 0.f;
    }
}

static int grid_for(int64_t n, int threads) {
    return (int)std::max<int64_t>(1, std::min<int64_t>(cdiv(n, threads), (int64_t)sm_count() * 16));
}

// ---- mixed precision: FP16 OTF with a power-of-two scale per kz plane -------

// max |OTF|^2 over plane kz (one CTA per plane, FP32: only the exponent is used)
__global__ void k_otf_plane_max(const float2* __restrict__ otf, int64_t Fy, int64_t Hx, int64_t P,
                                float* __restrict__ inv) {
    const int64_t kz = blockIdx.x;
    const float2* pl = otf + kz * Fy * P;
    float m = 0.f;
    for (int64_t i = threadIdx.x; i < Fy * Hx; i += blockDim.x) {
        const int64_t ky = i / Hx, kx = i - ky * Hx;
        const float2 v = pl[ky * P + kx];
        m = fmaxf(m, v.x * v.x + v.y * v.y);
    }
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
    __shared__ float red[32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmaxf(m, red[w]);
        m = fmaxf(m, red[0]);
        // |OTF| < 2^e with e = ceil(log2 sqrt(m)); scaled values stay below 2^14
        int e = 0;
        if (m > 0.f) {
            frexpf(sqrtf(m), &e);
        }
        inv[kz] = ldexpf(1.f, e - 14);  // OTF = stored * inv
    }
}

__global__ void k_otf_to_half(const float2* __restrict__ otf, int64_t n_plane, int64_t n,
                              const float* __restrict__ inv, __half2* __restrict__ out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float s = 1.f / inv[i / n_plane];  // power of two: exact
        const float2 v = otf[i];
        out[i] = __floats2half2_rn(v.x * s, v.y * s);
    }
}

int quantize_otf(const ConvPlan& p, cudaStream_t s) {
    const int64_t Fz = p.F[0], Fy = p.F[1];
    k_otf_plane_max<<<(unsigned)Fz, 256, 0, s>>>(p.otf, Fy, p.Hx, p.P, p.otf_inv);
    DK_LAUNCHED();
    const int64_t n = Fz * Fy * p.P;
    k_otf_to_half<<<grid_for(n, 256), 256, 0, s>>>(p.otf, Fy * p.P, n, p.otf_inv, p.otf16);
    DK_LAUNCHED();
    return DECON_OK;
}

}  // namespace dk

using namespace dk;

extern "C" {

const char* decon_last_error(void) { return g_err.c_str(); }

int decon_version(void) { return 100; }

int64_t decon_launch_count(void) { return (int64_t)g_launches.load(); }

int64_t decon_next_smooth(int64_t n) {
    int64_t m = n < 1 ? 1 : n;
    for (;; ++m) {
        int64_t r = m;
        for (int p : {2, 3, 5})
            while (r % p == 0) r /= p;
        if (r == 1) return m;
    }
}

int decon_fast_padded_shape(int ndim, const int64_t* signal, const int64_t* kernel,
                            const int64_t* pad, int64_t* out) {
    if (!signal || !kernel || !out) return fail(DECON_ERR_NULL, "null pointer");
    for (int i = 0; i < ndim; ++i) {
        const int64_t need = (pad && pad[i] >= 0) ? pad[i] : kernel[i] - 1;
        out[i] = decon_next_smooth(std::max(signal[i] + need, kernel[i]));
    }
    return DECON_OK;
}

// Kernel sum (FP64, linops_mlx.py:408-409) and OTF = rfftn(kernel canvas):
// X pass over all Fz*Fy rows straight into the OTF buffer, then in-place Y
// and Z forward passes (unpruned); operator_norm_sq = max |OTF|^2.  Reads
// the two FP64 scalars back (synchronises the stream).
static int build_otf(decon_conv* p, const float* kernel, int normalize, cudaStream_t s) {
    int st;
    const int64_t Fz = p->F[0], Fy = p->F[1];
    p->kdiv = 1.f;
    const int64_t nk = p->K[0] * p->K[1] * p->K[2];
    if (normalize) {
        DK_TRY(reduce_f32(kernel, nullptr, nk, DECON_RED_SUM, p->dscal, p->partials, p->npartials, s));
        double ksum = 0;
        cudaError_t e = cudaMemcpyAsync(&ksum, p->dscal, sizeof(double), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return fail(DECON_ERR_CUDA, "kernel sum failed: %s", cudaGetErrorString(e));
        p->kdiv = (float)ksum;
    }
    Win3 none{0, 0, 0, 0, 0, 0};
    if ((st = launch_xr2c(*p, PRO_KERNEL, kernel, none, 0.f, 0.f, Fz, p->otf, s)) ||
        (st = launch_col(*p, p->ax_y, p->T_y, COL_FWD, p->otf, Fy * p->P, p->P, (int)Fy, p->otf,
                         Fy * p->P, p->P, (int)Fy, Fz, s)) ||
        (st = launch_col(*p, p->ax_z, p->T_z, COL_FWD, p->otf, p->P, Fy * p->P, (int)Fz, p->otf,
                         p->P, Fy * p->P, (int)Fz, Fy, s)) ||
        (st = max_abs2(p->otf, Fz * Fy, p->Hx, p->P, p->dscal + 1, p->partials, s)))
        return st;
    double nrm = 0;
    cudaError_t e = cudaMemcpyAsync(&nrm, p->dscal + 1, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(DECON_ERR_CUDA, "OTF build failed: %s", cudaGetErrorString(e));
    p->norm_sq = nrm;
    if (p->precision == 1) DK_TRY(quantize_otf(*p, s));
    DK_TRY(build_otf_kmajor(*p, s));
    return DECON_OK;
}

static int conv_create_impl(const float* kernel, const int64_t kshape[3],
                            const int64_t signal_shape[3], const int64_t fft_shape[3], int normalize,
                            bool circular, void* stream, decon_conv** out) {
    if (!kernel || !kshape || !signal_shape || !fft_shape || !out)
        return fail(DECON_ERR_NULL, "decon_conv_create: null pointer");
    *out = nullptr;
    for (int i = 0; i < 3; ++i) {
        if (kshape[i] < 1 || signal_shape[i] < 1)
            return fail(DECON_ERR_VALUE, "shapes must be positive");
        const int64_t need = signal_shape[i] + kshape[i] - 1;
        if (!circular && fft_shape[i] < need)
            return fail(DECON_ERR_VALUE,
                        "fft_shape (%lld, %lld, %lld) is too small for linear convolution; "
                        "minimum is (%lld, %lld, %lld)",
                        (long long)fft_shape[0], (long long)fft_shape[1], (long long)fft_shape[2],
                        (long long)(signal_shape[0] + kshape[0] - 1),
                        (long long)(signal_shape[1] + kshape[1] - 1),
                        (long long)(signal_shape[2] + kshape[2] - 1));
    }
    decon_conv* p = new (std::nothrow) decon_conv();
    if (!p) return fail(DECON_ERR_OOM, "host allocation failed");
    for (int i = 0; i < 3; ++i) {
        p->N[i] = signal_shape[i];
        p->F[i] = fft_shape[i];
        p->K[i] = kshape[i];
    }
    cudaGetDevice(&p->device);
    const int64_t Fz = p->F[0], Fy = p->F[1], Fx = p->F[2];
    p->odd = (int)(Fx & 1);
    p->Hx = Fx / 2 + 1;
    p->P = round_up(p->Hx, 16);
    const int Lx = p->odd ? (int)Fx : (int)(Fx / 2);
    if (Lx > kSmemElems || Fy > kSmemElems || Fz > kSmemElems) {
        delete p;
        return fail(DECON_ERR_UNSUPPORTED, "FFT axis longer than %d points is not supported",
                    kSmemElems);
    }
    if (!plan_axis(Lx, p->ax_x) || !plan_axis((int)Fy, p->ax_y) || !plan_axis((int)Fz, p->ax_z)) {
        delete p;
        return fail(DECON_ERR_UNSUPPORTED,
                    "fft_shape (%lld, %lld, %lld): every axis must factor into 2, 3, 5 and 7",
                    (long long)Fz, (long long)Fy, (long long)Fx);
    }
    p->T_x = 0;
    // lines per CTA
    {
        p->T_x = p->T_x0 = fft_lines_per_cta(p->ax_x, 32);
        p->T_y = p->T_y0 = fft_lines_per_cta(p->ax_y, 16);
        p->T_z = p->T_z0 = fft_lines_per_cta(p->ax_z, 16);
    }
    int st;
    const cudaStream_t s = as_stream(stream);
    const int64_t nz = p->N[0], ny = p->N[1];
    if ((st = make_twiddles((int)Fx, &p->twx)) || (st = make_twiddles((int)Fy, &p->twy)) ||
        (st = make_twiddles((int)Fz, &p->twz))) {
        free_plan(p);
        delete p;
        return st;
    }
    p->ax_x.tw = p->twx;
    p->ax_x.tws = p->odd ? 1 : 2;
    p->ax_y.tw = p->twy;
    p->ax_y.tws = 1;
    p->ax_z.tw = p->twz;
    p->ax_z.tws = 1;
    p->npartials = std::max<int64_t>(reduce_partials_needed(), cdiv(nz * ny, p->T_x) + 1);
    if ((st = dev_alloc((void**)&p->otf, (size_t)Fz * Fy * p->P * sizeof(float2), "OTF")) ||
        (st = dev_alloc((void**)&p->s1, (size_t)nz * ny * p->P * sizeof(float2), "spectrum S1")) ||
        (st = dev_alloc((void**)&p->s2, (size_t)nz * Fy * p->P * sizeof(float2), "spectrum S2")) ||
        (st = dev_alloc((void**)&p->dscal, 16 * sizeof(double), "scalars")) ||
        (st = dev_alloc((void**)&p->partials, p->npartials * sizeof(double), "partials"))) {
        free_plan(p);
        delete p;
        return st;
    }
    // fused Y / axial pass (opt-in, DECON_YZ=1): the kx-major OTF copy now;
    // otherwise decon_conv_set_schedule allocates it on request
    if (!circular && yz_supported(p->N, p->F) && getenv("DECON_YZ") != nullptr &&
        getenv("DECON_NO_YZ") == nullptr &&
        (st = dev_alloc((void**)&p->otft, (size_t)p->Hx * Fy * Fz * sizeof(float2), "kx-major OTF"))) {
        free_plan(p);
        delete p;
        return st;
    }
    // TMA tensor maps for the strided column passes (power-of-two lengths
    // <= 512, 16-column tiles).  DECON_NO_TMA=1 selects the plain-load kernels.
    {
        const bool allow = getenv("DECON_NO_TMA") == nullptr;
        const int64_t P = p->P;
        p->s1_box = (int)std::min<int64_t>(ny, 256);
        p->s2y_box = (int)std::min<int64_t>(Fy, 256);
        p->s2z_box = (int)std::min<int64_t>(nz, 256);
        p->otf_box = (int)std::min<int64_t>(Fz, 256);
        p->tma_y = allow && tma_length_ok(p->ax_y.L) && p->T_y == 16 &&
                   encode_spectrum_map(&p->tm_s1_j1, p->s1, P, ny, nz, p->s1_box, 1) &&
                   encode_spectrum_map(&p->tm_s2_j1, p->s2, P, Fy, nz, p->s2y_box, 1);
        p->tma_z = allow && tma_length_ok(p->ax_z.L) && p->T_z == 16 &&
                   encode_spectrum_map(&p->tm_s2_j2, p->s2, P, Fy, nz, 1, p->s2z_box) &&
                   encode_spectrum_map(&p->tm_otf_z, p->otf, P, Fy, Fz, 1, p->otf_box);
    }
    if ((st = build_otf(p, kernel, normalize, s))) {
        free_plan(p);
        delete p;
        return st;
    }
    *out = p;
    return DECON_OK;
}

int decon_conv_create(const float* kernel, const int64_t kshape[3], const int64_t signal_shape[3],
                      const int64_t fft_shape[3], int normalize, void* stream, decon_conv** out) {
    return conv_create_impl(kernel, kshape, signal_shape, fft_shape, normalize, false, stream, out);
}

int decon_conv_create_circular(const float* kernel, const int64_t shape[3], int normalize,
                               void* stream, decon_conv** out) {
    return conv_create_impl(kernel, shape, shape, shape, normalize, true, stream, out);
}

int decon_conv_set_kernel(decon_conv* p, const float* kernel, int normalize, void* stream) {
    if (!p || !kernel) return fail(DECON_ERR_NULL, "decon_conv_set_kernel: null pointer");
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != p->device)
        return fail(DECON_ERR_VALUE, "decon_conv_set_kernel: plan lives on device %d, current is %d",
                    p->device, cur);
    return build_otf(p, kernel, normalize, as_stream(stream));
}

int decon_conv_set_precision(decon_conv* p, int precision, void* stream) {
    if (!p) return fail(DECON_ERR_NULL, "decon_conv_set_precision: null plan");
    if (precision != 0 && precision != 1)
        return fail(DECON_ERR_VALUE, "precision must be 0 (FP32) or 1 (FP16 OTF), got %d", precision);
    if (precision == 0) {
        p->precision = 0;
        return DECON_OK;
    }
    if (!zpass_pipelined(*p))
        return fail(DECON_ERR_UNSUPPORTED,
                    "mixed precision needs the pipelined axial pass (Fz in {64, 256}, or 128 with "
                    "Nz <= 64); this plan has Fz = %lld, Nz = %lld",
                    (long long)p->F[0], (long long)p->N[0]);
    const int64_t n = p->F[0] * p->F[1] * p->P;
    int st;
    if (!p->otf16 && (st = dev_alloc((void**)&p->otf16, (size_t)n * sizeof(__half2), "FP16 OTF"))) return st;
    if (!p->otf_inv && (st = dev_alloc((void**)&p->otf_inv, (size_t)p->F[0] * sizeof(float), "OTF scales")))
        return st;
    DK_TRY(quantize_otf(*p, as_stream(stream)));
    if (!p->tma_otf16)
        p->tma_otf16 = encode_half_plane_map(&p->tm_otf16_z, p->otf16, p->P, p->F[1], p->F[0], p->otf_box);
    p->precision = 1;
    return DECON_OK;
}

int decon_conv_destroy(decon_conv* p) {
    if (!p) return DECON_OK;
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != p->device) cudaSetDevice(p->device);
    free_plan(p);
    if (cur != p->device) cudaSetDevice(cur);
    delete p;
    return DECON_OK;
}

int decon_conv_set_schedule(decon_conv* p, int sched) {
    if (!p) return fail(DECON_ERR_NULL, "null plan");
    if (sched < 0 || sched > 63) return fail(DECON_ERR_VALUE, "schedule bits out of range: %d", sched);
    // radix plans and lines per CTA of the runtime-length axes; the twiddle
    // tables depend on the length only and stay
    const int order = (sched & DECON_SCHED_ODD_RADIX) ? 1 : 0;
    Axis* axes[3] = {&p->ax_x, &p->ax_y, &p->ax_z};
    int* lines[3] = {&p->T_x, &p->T_y, &p->T_z};
    const int lines0[3] = {p->T_x0, p->T_y0, p->T_z0};
    for (int i = 0; i < 3; ++i) {
        Axis a;
        const int L = axes[i]->L;
        if (!plan_axis(L, a, order)) return fail(DECON_ERR_UNSUPPORTED, "radix plan failed");
        a.tw = axes[i]->tw;
        a.tws = axes[i]->tws;
        *axes[i] = a;
        const bool runtime = !static_length(L);
        *lines[i] = (runtime && (sched & DECON_SCHED_HALF_LINES) && lines0[i] >= 2) ? lines0[i] / 2
                                                                                  : lines0[i];
    }
    if ((sched & DECON_SCHED_FUSED) && !p->otft && yz_supported(p->N, p->F) && p->F[0] != p->N[0]) {
        // the fused pass needs the kx-major OTF copy: allocate and fill it
        DK_TRY(dev_alloc((void**)&p->otft, (size_t)p->Hx * p->F[1] * p->F[0] * sizeof(float2),
                         "kx-major OTF"));
        cudaStream_t s = nullptr;
        DK_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        const int e = build_otf_kmajor(*p, s);
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
        DK_TRY(e);
    }
    p->sched = sched;
    return DECON_OK;
}

int decon_conv_get_schedule(const decon_conv* p, int* sched) {
    if (!p || !sched) return fail(DECON_ERR_NULL, "null pointer");
    *sched = p->sched;
    return DECON_OK;
}

int decon_conv_fused_yz(const decon_conv* p, int* out) {
    if (!p || !out) return fail(DECON_ERR_NULL, "null pointer");
    *out = use_yz(*p) ? 1 : 0;
    return DECON_OK;
}

int decon_conv_norm_sq(const decon_conv* p, double* out) {
    if (!p || !out) return fail(DECON_ERR_NULL, "null pointer");
    *out = p->norm_sq;
    return DECON_OK;
}

int decon_conv_shape(const decon_conv* p, int64_t fft_shape[3], int64_t* pitch) {
    if (!p) return fail(DECON_ERR_NULL, "null plan");
    if (fft_shape)
        for (int i = 0; i < 3; ++i) fft_shape[i] = p->F[i];
    if (pitch) *pitch = p->P;
    return DECON_OK;
}

int decon_conv_get_otf(const decon_conv* p, float* out, void* stream) {
    if (!p || !out) return fail(DECON_ERR_NULL, "null pointer");
    DK_CUDA(cudaMemcpy2DAsync(out, p->Hx * sizeof(float2), p->otf, p->P * sizeof(float2),
                              p->Hx * sizeof(float2), p->F[0] * p->F[1], cudaMemcpyDeviceToDevice,
                              as_stream(stream)));
    return DECON_OK;
}

int decon_conv_forward(decon_conv* p, const float* x, float* y, void* stream) {
    if (!p || !x || !y) return fail(DECON_ERR_NULL, "null pointer");
    const cudaStream_t s = as_stream(stream);
    const Win3 w = full_window(p->N);
    DK_TRY(spectrum_forward(*p, PRO_ARRAY, x, w, 0.f, 0.f, s));
    DK_TRY(spectrum_filter_back(*p, false, s));
    DK_TRY(launch_xc2r(*p, EPI_STORE, p->s1, w, y, nullptr, nullptr, 0.f, nullptr, nullptr, s));
    return DECON_OK;
}

// compose(FractionalAreaDownsample(2), LinearFFTConvolver) in one pass
// sequence: the 2x area sum of the convolution is the X C2R epilogue, its
// adjoint the X R2C prologue (core_operators.py:222-352 with unit weights).
static bool down2_ok(const decon_conv* p) {
    return !p->odd && !((p->N[0] | p->N[1] | p->N[2]) & 1);
}

int decon_conv_forward_down2(decon_conv* p, const float* x, float* y, void* stream) {
    if (!p || !x || !y) return fail(DECON_ERR_NULL, "null pointer");
    if (!down2_ok(p))
        return fail(DECON_ERR_UNSUPPORTED, "decon_conv_forward_down2: extents must be even (and Fx)");
    const cudaStream_t s = as_stream(stream);
    const Win3 w = full_window(p->N);
    DK_TRY(spectrum_forward(*p, PRO_ARRAY, x, w, 0.f, 0.f, s));
    DK_TRY(spectrum_filter_back(*p, false, s));
    DK_TRY(launch_xc2r(*p, EPI_DOWN2, p->s1, w, y, nullptr, nullptr, 0.f, nullptr, nullptr, s));
    return DECON_OK;
}

int decon_conv_adjoint_up2(decon_conv* p, const float* y, float* x, void* stream) {
    if (!p || !x || !y) return fail(DECON_ERR_NULL, "null pointer");
    if (!down2_ok(p))
        return fail(DECON_ERR_UNSUPPORTED, "decon_conv_adjoint_up2: extents must be even (and Fx)");
    const cudaStream_t s = as_stream(stream);
    const Win3 w = full_window(p->N);
    DK_TRY(spectrum_forward(*p, PRO_UP2, y, w, 0.f, 0.f, s));
    DK_TRY(spectrum_filter_back(*p, true, s));
    DK_TRY(launch_xc2r(*p, EPI_STORE, p->s1, w, x, nullptr, nullptr, 0.f, nullptr, nullptr, s));
    return DECON_OK;
}

int decon_conv_adjoint(decon_conv* p, const float* y, float* x, void* stream) {
    if (!p || !x || !y) return fail(DECON_ERR_NULL, "null pointer");
    const cudaStream_t s = as_stream(stream);
    const Win3 w = full_window(p->N);
    DK_TRY(spectrum_forward(*p, PRO_ARRAY, y, w, 0.f, 0.f, s));
    DK_TRY(spectrum_filter_back(*p, true, s));
    DK_TRY(launch_xc2r(*p, EPI_STORE, p->s1, w, x, nullptr, nullptr, 0.f, nullptr, nullptr, s));
    return DECON_OK;
}

int decon_rl_setup(decon_conv* p, const float* observed, float background, const float* x_init,
                   float* x, float* sens, void* stream) {
    if (!p || !observed || !x || !sens) return fail(DECON_ERR_NULL, "null pointer");
    const cudaStream_t s = as_stream(stream);
    const Win3 w = full_window(p->N);
    const int64_t n = p->N[0] * p->N[1] * p->N[2];
    // sens_raw = A^T 1 (rl_mlx.py:129)
    DK_TRY(spectrum_forward(*p, PRO_CONST, nullptr, w, 1.f, 0.f, s));
    DK_TRY(spectrum_filter_back(*p, true, s));
    DK_TRY(launch_xc2r(*p, EPI_STORE, p->s1, w, sens, nullptr, nullptr, 0.f, nullptr, nullptr, s));
    if (x_init) {
        if (x_init != x) DK_CUDA(cudaMemcpyAsync(x, x_init, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
    } else {
        // x0 = A^T max(y - b, 1e-6) (rl_mlx.py:123-125)
        DK_TRY(spectrum_forward(*p, PRO_RLINIT, observed, w, 0.f, background, s));
        DK_TRY(spectrum_filter_back(*p, true, s));
        DK_TRY(launch_xc2r(*p, EPI_STORE, p->s1, w, x, nullptr, nullptr, 0.f, nullptr, nullptr, s));
    }
    DK_TRY(reduce_f32(sens, nullptr, n, DECON_RED_MAX, p->dscal + 2, p->partials, p->npartials, s));
    k_rl_mask<<<grid_for(n, 256), 256, 0, s>>>(x, sens, p->dscal + 2, n, 1);
    DK_LAUNCHED();
    DK_CUDA(cudaStreamSynchronize(s));
    return DECON_OK;
}

int decon_rl_iteration(decon_conv* p, const float* observed, float background, const float* sens,
                       float* x, float* ratio, double* loss_sum, void* stream) {
    if (!p || !observed || !sens || !x || !ratio) return fail(DECON_ERR_NULL, "null pointer");
    const cudaStream_t s = as_stream(stream);
    const Win3 w = full_window(p->N);
    int nblk = 0;
    DK_TRY(spectrum_forward(*p, PRO_ARRAY, x, w, 0.f, 0.f, s));
    DK_TRY(spectrum_filter_back(*p, false, s));
    DK_TRY(launch_xc2r(*p, EPI_RL_RATIO, p->s1, w, ratio, observed, nullptr, background,
                       loss_sum ? p->partials : nullptr, &nblk, s));
    if (loss_sum) DK_TRY(finish_partials(p->partials, nblk, loss_sum, s));
    DK_TRY(spectrum_forward(*p, PRO_ARRAY, ratio, w, 0.f, 0.f, s));
    DK_TRY(spectrum_filter_back(*p, true, s));
    DK_TRY(launch_xc2r(*p, EPI_RL_UPDATE, p->s1, w, x, x, sens, 0.f, nullptr, nullptr, s));
    return DECON_OK;
}

int decon_rl_predict(decon_conv* p, const float* observed, float background, const float* x,
                     float* pred, double* loss_sum, void* stream) {
    if (!p || !observed || !x || !pred) return fail(DECON_ERR_NULL, "null pointer");
    const cudaStream_t s = as_stream(stream);
    const Win3 w = full_window(p->N);
    int nblk = 0;
    DK_TRY(spectrum_forward(*p, PRO_ARRAY, x, w, 0.f, 0.f, s));
    DK_TRY(spectrum_filter_back(*p, false, s));
    DK_TRY(launch_xc2r(*p, EPI_PRED, p->s1, w, pred, observed, nullptr, background,
                       loss_sum ? p->partials : nullptr, &nblk, s));
    if (loss_sum) DK_TRY(finish_partials(p->partials, nblk, loss_sum, s));
    return DECON_OK;
}

}  // extern "C"
