// Widefield PSF synthesis on the device: PSF(z) = |IFFT2(P(kx, ky) e^{2 pi i kz z})|^2.
//
// Replaces the NumPy loop of deconlib's pupil_to_psf (psf/widefield.py:18-73)
// with two FFT passes per chunk of z planes, built on the library's own
// shared-memory FFT engine:
//
//   pass 1 (k_psf_cols): defocus P(ky, kx) e^{2 pi i kz z} on load (phase in
//     FP64 with sincospi; pupil and kz are re-read per plane from L2), inverse
//     FFT along y over tiles of T columns, complex planes written to scratch;
//   pass 2 (k_psf_rows): inverse FFT along x over T contiguous rows, intensity
//     |.|^2 times the final scale, written straight into the PSF.
//
// 20 bytes of HBM traffic per voxel (complex write + read, float write).  The
// unit-sum normalisation needs no pass over the PSF: |e^{i phi}| = 1, so by
// Parseval every plane's unnormalised intensity sums to ny nx sum|P|^2, and
// the total is nz ny nx sum|P|^2, an FP64 reduction over the pupil alone
// (k_psf_energy).  numpy's ifft2 divides by ny nx; without normalisation the
// PSF carries that factor squared.
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <vector>

#include "conv_impl.cuh"

namespace dk {

// Complex scratch per chunk of planes: at most this many voxels (256 MB), or
// one plane when a plane is larger.
constexpr int64_t kPsfChunkVoxels = int64_t(1) << 25;
constexpr int kPsfEnergyBlocks = 256;

struct PsfColArgs {
    const float2* pupil;
    const double* kz;
    const double* z;  // this chunk's first plane
    float2* a;
    int64_t nyx;
    int nx, ntiles, T;
    Axis ax;  // y axis, L = ny
};

struct PsfRowArgs {
    const float2* a;
    float* psf;  // this chunk's first plane
    int64_t nrows;
    int T;
    FastDiv fd_L;
    Axis ax;               // x axis, L = nx
    const double* energy;  // sum |P|^2 (normalize) or nullptr
    double norm_div;       // nz ny nx (normalize)
    float fixed_scale;     // 1 / (ny nx)^2 (no normalisation)
};

// sum |P|^2 in FP64, one partial per CTA
__global__ void k_psf_energy(const float2* __restrict__ pupil, int64_t n, double* __restrict__ partials) {
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float2 v = pupil[i];
        acc += (double)v.x * v.x + (double)v.y * v.y;
    }
    const double s = block_sum(acc);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

// Pass 1: one CTA = T columns of one plane; defocus on load, inverse FFT along y.
template <int LS>
__global__ void __launch_bounds__(LS > 0 ? kFftThreads : kDynThreads, 1) k_psf_cols(const PsfColArgs a) {
    extern __shared__ float2 sm[];
    const int T = a.T, L = a.ax.L, tid = threadIdx.x;
    const int64_t o = blockIdx.x / a.ntiles;
    const int x0 = (int)(blockIdx.x - o * a.ntiles) * T;
    const double zz = a.z[o];
    const int lgT = 31 - __clz(T);  // T is a power of two
    for (int q = tid; q < L * T; q += blockDim.x) {
        const int j = q >> lgT, t = q & (T - 1);
        float2 v = make_float2(0.f, 0.f);
        if (x0 + t < a.nx) {
            const int64_t p = (int64_t)j * a.nx + x0 + t;
            double sn, cs;
            sincospi(2.0 * a.kz[p] * zz, &sn, &cs);
            const float2 pv = a.pupil[p];
            v = make_float2((float)((double)pv.x * cs - (double)pv.y * sn),
                            (float)((double)pv.x * sn + (double)pv.y * cs));
        }
        sm[phys(j, t, T)] = v;
    }
    __syncthreads();
    fft_lines<+1, LS>(sm, T, tid % T, tid / T, a.ax);
    float2* dst = a.a + o * a.nyx + x0;
    for (int q = tid; q < L * T; q += blockDim.x) {
        const int j = q >> lgT, t = q & (T - 1);
        if (x0 + t < a.nx) dst[(int64_t)j * a.nx + t] = sm[phys(j, t, T)];
    }
}

// Pass 2: one CTA = T contiguous rows; inverse FFT along x, |.|^2 * scale.
template <int LS>
__global__ void __launch_bounds__(LS > 0 ? kFftThreads : kDynThreads, 1) k_psf_rows(const PsfRowArgs a) {
    extern __shared__ float2 sm[];
    const int T = a.T, L = a.ax.L, tid = threadIdx.x;
    const int64_t row0 = (int64_t)blockIdx.x * T;
    const int64_t left = a.nrows - row0;
    const int nr = left < T ? (int)left : T;
    const float2* src = a.a + row0 * L;
    for (int q = tid; q < T * L; q += blockDim.x) {
        const int t = fdiv(q, a.fd_L), j = q - t * L;
        sm[phys(j, t, T)] = t < nr ? src[q] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    fft_lines<+1, LS>(sm, T, tid % T, tid / T, a.ax);
    float scale = a.fixed_scale;
    if (a.energy) {
        const double tot = a.norm_div * *a.energy;
        scale = tot > 0.0 ? (float)(1.0 / tot) : 1.f;
    }
    float* dst = a.psf + row0 * L;
    for (int q = tid; q < nr * L; q += blockDim.x) {
        const int t = fdiv(q, a.fd_L), j = q - t * L;
        const float2 v = sm[phys(j, t, T)];
        dst[q] = (v.x * v.x + v.y * v.y) * scale;
    }
}

// Twiddle tables W_L^m = exp(-2 pi i m / L) per (device, L), kept for the
// life of the process (the first call for a length uploads it and waits for
// the copy, so every stream may read the table).
static int psf_twiddles(int L, const float2** out) {
    static std::mutex mu;
    static std::map<std::pair<int, int>, float2*> cache;
    int dev = 0;
    DK_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    float2*& t = cache[std::make_pair(dev, L)];
    if (!t) {
        std::vector<float2> h(L);
        for (int m = 0; m < L; ++m) {
            const double ang = -2.0 * M_PI * (double)m / (double)L;
            h[m] = make_float2((float)std::cos(ang), (float)std::sin(ang));
        }
        float2* d = nullptr;
        DK_CUDA(cudaMalloc(&d, h.size() * sizeof(float2)));
        if (upload_blocking(d, h.data(), h.size() * sizeof(float2)) != DECON_OK) {
            cudaFree(d);
            return fail(DECON_ERR_CUDA, "decon_pupil_to_psf: twiddle upload failed");
        }
        t = d;
    }
    *out = t;
    return DECON_OK;
}

// Stream-ordered scratch from a per-device pool that keeps up to 1 GB
// reserved between calls (no re-mapping of the chunk buffer on every call).
static int psf_pool(cudaMemPool_t* out) {
    static std::mutex mu;
    static std::map<int, cudaMemPool_t> pools;
    int dev = 0;
    DK_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    auto it = pools.find(dev);
    if (it == pools.end()) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool;
        DK_CUDA(cudaMemPoolCreate(&pool, &props));
        uint64_t keep = uint64_t(1) << 30;
        DK_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
        it = pools.emplace(dev, pool).first;
    }
    *out = it->second;
    return DECON_OK;
}


static int threads_for_lines(int T, const Axis& ax) {
    return std::max(64, (int)round_up((int64_t)T * ax.tpl, 32));
}

template <int LS>
static void* cols_ptr() { return (void*)k_psf_cols<LS>; }
template <int LS>
static void* rows_ptr() { return (void*)k_psf_rows<LS>; }

static void* pick(int L, bool cols) {
#define DK_CASE(n) \
    if (L == n) return cols ? cols_ptr<n>() : rows_ptr<n>();
    DK_STATIC_LENGTHS(DK_CASE)
#undef DK_CASE
    return cols ? cols_ptr<0>() : rows_ptr<0>();
}

static int launch_args(void* fn, int64_t nblk, int nthr, size_t smem, cudaStream_t st, void* args) {
    DK_TRY(kernel_prepare(fn, smem, nthr, nullptr));
    if (nblk > 0x7fffffffLL) return fail(DECON_ERR_UNSUPPORTED, "decon_pupil_to_psf: grid too large");
    void* params[] = {args};
    DK_CUDA(cudaLaunchKernel(fn, dim3((unsigned)nblk), dim3(nthr), params, smem, st));
    count_launch();
    return DECON_OK;
}

}  // namespace dk

using namespace dk;

extern "C" int decon_pupil_to_psf(const float* pupil, const double* kz, const double* z, int64_t nz,
                                  int64_t ny, int64_t nx, int normalize, float* psf, void* stream) {
    if (nz < 1 || ny < 1 || nx < 1) return fail(DECON_ERR_VALUE, "decon_pupil_to_psf: empty shape");
    if (!pupil || !kz || !z || !psf) return fail(DECON_ERR_NULL, "decon_pupil_to_psf: null pointer");
    if (ny > kSmemElems || nx > kSmemElems)
        return fail(DECON_ERR_UNSUPPORTED, "decon_pupil_to_psf: planes larger than %d points per axis",
                    kSmemElems);
    Axis axx, axy;
    if (!plan_axis((int)nx, axx) || !plan_axis((int)ny, axy))
        return fail(DECON_ERR_UNSUPPORTED,
                    "decon_pupil_to_psf: pupil shape (%lld, %lld) must factor into 2, 3, 5 and 7",
                    (long long)ny, (long long)nx);
    const cudaStream_t st = as_stream(stream);
    const int64_t nyx = ny * nx;
    const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(nz, kPsfChunkVoxels / nyx));
    const float2 *twx = nullptr, *twy = nullptr;
    DK_TRY(psf_twiddles((int)nx, &twx));
    DK_TRY(psf_twiddles((int)ny, &twy));
    axx.tw = twx;
    axy.tw = twy;
    axx.tws = axy.tws = 1;
    cudaMemPool_t pool;
    DK_TRY(psf_pool(&pool));
    float2* a = nullptr;
    double* red = nullptr;
    auto run = [&]() -> int {
        DK_CUDA(cudaMallocFromPoolAsync((void**)&a, (size_t)(chunk * nyx) * sizeof(float2), pool, st));
        const double inv_n = 1.0 / ((double)nx * (double)ny);
        PsfRowArgs ra{};
        ra.fixed_scale = (float)(inv_n * inv_n);
        if (normalize) {
            DK_CUDA(cudaMallocFromPoolAsync((void**)&red, (kPsfEnergyBlocks + 1) * sizeof(double), pool, st));
            const int nb = (int)std::min<int64_t>(kPsfEnergyBlocks, cdiv(nyx, 256));
            k_psf_energy<<<nb, 256, 0, st>>>(reinterpret_cast<const float2*>(pupil), nyx, red);
            DK_LAUNCHED();
            DK_TRY(finish_partials(red, nb, red + kPsfEnergyBlocks, st));
            ra.energy = red + kPsfEnergyBlocks;
            ra.norm_div = (double)nz * (double)nyx;
        }
        PsfColArgs ca{};
        ca.pupil = reinterpret_cast<const float2*>(pupil);
        ca.kz = kz;
        ca.a = a;
        ca.nyx = nyx;
        ca.nx = (int)nx;
        ca.ax = axy;
        ca.T = fft_lines_per_cta(axy, 32);
        ca.ntiles = (int)cdiv(nx, ca.T);
        ra.a = a;
        ra.ax = axx;
        ra.T = fft_lines_per_cta(axx, 32);
        ra.fd_L = make_fastdiv(nx);
        void* fc = pick((int)ny, true);
        void* fr = pick((int)nx, false);
        const int tc = threads_for_lines(ca.T, axy), tr = threads_for_lines(ra.T, axx);
        const size_t sc = (size_t)ca.T * ny * sizeof(float2), sr = (size_t)ra.T * nx * sizeof(float2);
        for (int64_t z0 = 0; z0 < nz; z0 += chunk) {
            const int64_t nzc = std::min(chunk, nz - z0);
            ca.z = z + z0;
            DK_TRY(launch_args(fc, nzc * ca.ntiles, tc, sc, st, &ca));
            ra.psf = psf + z0 * nyx;
            ra.nrows = nzc * ny;
            DK_TRY(launch_args(fr, cdiv(ra.nrows, ra.T), tr, sr, st, &ra));
        }
        return DECON_OK;
    };
    const int status = run();
    if (a) cudaFreeAsync(a, st);
    if (red) cudaFreeAsync(red, st);
    return status;
}
