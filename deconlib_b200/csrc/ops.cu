// Pad / crop, fractional-area resampling and finite-difference operators.
//
//   decon_window_copy      Pad and Crop, forward and adjoint (core_operators.py:29-137)
//   decon_band_weights     _banded_overlap_weights_1d (core_operators.py:151-202)
//   decon_banded_axis      _apply_banded_1d (core_operators.py:205-219)
//   decon_hessian3d_*      Hessian3D (linops_mlx.py:182-262, linops_core_mlx.py:42-80)
//   decon_gradient3d_*     Gradient3D (linops_mlx.py:92-122, linops_core_mlx.py:25-39)
//
// The stencils evaluate each difference in the same float32 operation order
// as the reference so results agree to the last few ulps.
#include <cmath>
#include <vector>

#include "conv_impl.cuh"
#include "stencil.cuh"
#include "zwalk.cuh"

namespace dk {

static int grid1d(int64_t n, int threads) {
    return (int)std::max<int64_t>(1, std::min<int64_t>(cdiv(n, threads), (int64_t)sm_count() * 32));
}

struct Box4 {
    int64_t ss[4], s0[4], ds[4], d0[4], ext[4];
};

__global__ void k_window_copy(const float* __restrict__ src, float* __restrict__ dst, Box4 b,
                              int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        int64_t r = i, c[4];
#pragma unroll
        for (int d = 3; d >= 0; --d) {
            c[d] = r % b.ds[d];
            r /= b.ds[d];
        }
        bool in = true;
        int64_t si = 0;
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            const int64_t k = c[d] - b.d0[d];
            in = in && k >= 0 && k < b.ext[d];
            si = si * b.ss[d] + (b.s0[d] + k);
        }
        dst[i] = in ? __ldg(src + si) : 0.f;
    }
}

// out[o, j, q] = sum_k w[j, k] in[o, idx[j, k], q], products rounded before
// the in-order sum as mx.sum(gathered * weight, -1) does (no FMA contraction).
// Resampled axis not innermost: one CTA row per (j, o), threads along q.
__global__ void k_banded_inner(const float* __restrict__ in, float* __restrict__ out, int64_t outer,
                               int64_t n_in, int64_t inner, int64_t n_out,
                               const int32_t* __restrict__ idx, const float* __restrict__ w,
                               int width) {
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= inner) return;
    const int64_t j = blockIdx.y;
    const int32_t* ij = idx + j * width;
    const float* wj = w + j * width;
    for (int64_t o = blockIdx.z; o < outer; o += gridDim.z) {
        const float* base = in + o * n_in * inner + q;
        float acc = 0.f;
        for (int k = 0; k < width; ++k)
            acc = __fadd_rn(acc, __fmul_rn(__ldg(wj + k), __ldg(base + (int64_t)__ldg(ij + k) * inner)));
        out[(o * n_out + j) * inner + q] = acc;
    }
}

// inner % 4 == 0 and 16-byte aligned rows: four neighbouring columns per
// thread as float4 (same per-element float operations as k_banded_inner).
__global__ void k_banded_inner4(const float* __restrict__ in, float* __restrict__ out, int64_t outer,
                                int64_t n_in, int64_t inner, int64_t n_out,
                                const int32_t* __restrict__ idx, const float* __restrict__ w,
                                int width) {
    const int64_t q4 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t inner4 = inner >> 2;
    if (q4 >= inner4) return;
    const int64_t j = blockIdx.y;
    const int32_t* ij = idx + j * width;
    const float* wj = w + j * width;
    for (int64_t o = blockIdx.z; o < outer; o += gridDim.z) {
        const float4* base = reinterpret_cast<const float4*>(in + o * n_in * inner) + q4;
        float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int k = 0; k < width; ++k) {
            const float wk = __ldg(wj + k);
            const float4 v = __ldg(base + (int64_t)__ldg(ij + k) * inner4);
            acc.x = __fadd_rn(acc.x, __fmul_rn(wk, v.x));
            acc.y = __fadd_rn(acc.y, __fmul_rn(wk, v.y));
            acc.z = __fadd_rn(acc.z, __fmul_rn(wk, v.z));
            acc.w = __fadd_rn(acc.w, __fmul_rn(wk, v.w));
        }
        reinterpret_cast<float4*>(out + (o * n_out + j) * inner)[q4] = acc;
    }
}

// Resampled axis innermost with at most kBandW taps: a thread keeps its
// output's taps and weights in registers and walks many rows.
constexpr int kBandW = 8;
__global__ void k_banded_last_rows(const float* __restrict__ in, float* __restrict__ out, int64_t outer,
                                   int64_t n_in, int64_t n_out, const int32_t* __restrict__ idx,
                                   const float* __restrict__ w, int width) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n_out) return;
    int32_t ij[kBandW];
    float wj[kBandW];
#pragma unroll
    for (int k = 0; k < kBandW; ++k) {
        ij[k] = k < width ? __ldg(idx + j * width + k) : 0;
        wj[k] = k < width ? __ldg(w + j * width + k) : 0.f;
    }
    // rows are independent: unrolled so that several rows' gathers are in flight
#pragma unroll 4
    for (int64_t o = blockIdx.y; o < outer; o += gridDim.y) {
        const float* base = in + o * n_in;
        float acc = 0.f;
#pragma unroll
        for (int k = 0; k < kBandW; ++k)
            if (k < width) acc = __fadd_rn(acc, __fmul_rn(wj[k], __ldg(base + ij[k])));
        out[o * n_out + j] = acc;
    }
}

// Resampled axis innermost (inner == 1): threads along the output axis.
__global__ void k_banded_last(const float* __restrict__ in, float* __restrict__ out, int64_t outer,
                              int64_t n_in, int64_t n_out, const int32_t* __restrict__ idx,
                              const float* __restrict__ w, int width) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n_out) return;
    const int32_t* ij = idx + j * width;
    const float* wj = w + j * width;
    for (int64_t o = blockIdx.y; o < outer; o += gridDim.y) {
        const float* base = in + o * n_in;
        float acc = 0.f;
        for (int k = 0; k < width; ++k)
            acc = __fadd_rn(acc, __fmul_rn(__ldg(wj + k), __ldg(base + __ldg(ij + k))));
        out[o * n_out + j] = acc;
    }
}

// ---- finite differences, Neumann boundary ----------------------------------

struct Vol {
    const float* p;
    int64_t nz, ny, nx;
    __device__ __forceinline__ float at(int64_t z, int64_t y, int64_t x) const {
        return __ldg(p + (z * ny + y) * nx + x);
    }
    __device__ __forceinline__ float operator()(int64_t z, int64_t y, int64_t x) const {
        return at(z, y, x);
    }
};

// Hessian3D.forward (linops_mlx.py:224-242): six weighted components, the z
// axis walked in registers (zwalk.cuh): each input value is loaded once per
// tile instead of once per tap and the outputs leave in rows of 32 (on the
// B200 57 vs 107 us for a per-voxel global-memory kernel at 128x256x256,
// bit-identical results).
template <class IDX>
__global__ void __launch_bounds__(256) k_hessian_fwd_z(const float* __restrict__ x, float* __restrict__ h,
                                                       Dims d, W6 w) {
    const IDX n = (IDX)(d.nz * d.ny * d.nx);
    hess_zwalk<IDX, 1>(
        d, w, [&](IDX i) { return __ldg(x + i); }, [](const float& r, int) { return r; },
        [&](IDX i, const float (*hv)[6]) {
#pragma unroll
            for (int c = 0; c < 6; ++c) h[c * n + i] = hv[0][c];
        });
}

__global__ void k_gradient_fwd(Vol f, float* __restrict__ g, float r) {
    const int64_t n = f.nz * f.ny * f.nx;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t x = i % f.nx, t = i / f.nx, y = t % f.ny, z = t / f.ny;
        const float c = f.at(z, y, x);
        g[i] = r * (f.at(clampi(z + 1, f.nz), y, x) - c);
        g[n + i] = f.at(z, clampi(y + 1, f.ny), x) - c;
        g[2 * n + i] = f.at(z, y, clampi(x + 1, f.nx)) - c;
    }
}

// d1_fwd_adj (linops_core_mlx.py:35-39): [-g0, g[i-1] - g[i], g[n-2]]
__device__ __forceinline__ float d1f_adj(const float* g, int64_t i, int64_t n, int64_t s, float sc) {
    if (n == 1) return -(__ldg(g) * sc);
    if (i == 0) return -(__ldg(g) * sc);
    if (i == n - 1) return __ldg(g + (n - 2) * s) * sc;
    return __ldg(g + (i - 1) * s) * sc - __ldg(g + i * s) * sc;
}

__global__ void k_gradient_adj(const float* __restrict__ g, float* __restrict__ out, int64_t nz,
                               int64_t ny, int64_t nx, float r) {
    const int64_t n = nz * ny * nx, sz = ny * nx, sy = nx;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t x = i % nx, t = i / nx, y = t % ny, z = t / ny;
        const float az = d1f_adj(g + y * sy + x, z, nz, sz, r);
        const float ay = d1f_adj(g + n + z * sz + x, y, ny, sy, 1.f);
        const float ax = d1f_adj(g + 2 * n + z * sz + y * sy, x, nx, 1, 1.f);
        out[i] = (az + ay) + ax;
    }
}

}  // namespace dk

using namespace dk;

extern "C" {

int decon_window_copy(const float* src, const int64_t* src_shape, const int64_t* src_start,
                      float* dst, const int64_t* dst_shape, const int64_t* dst_start,
                      const int64_t* ext, int ndim, void* stream) {
    if (!src || !dst || !src_shape || !dst_shape || !ext) return fail(DECON_ERR_NULL, "null pointer");
    if (ndim < 1 || ndim > 4) return fail(DECON_ERR_VALUE, "window copy supports 1-4 dims");
    Box4 b;
    const int off = 4 - ndim;
    int64_t n = 1;
    for (int d = 0; d < 4; ++d) {
        if (d < off) {
            b.ss[d] = b.ds[d] = b.ext[d] = 1;
            b.s0[d] = b.d0[d] = 0;
        } else {
            const int k = d - off;
            b.ss[d] = src_shape[k];
            b.ds[d] = dst_shape[k];
            b.ext[d] = ext[k];
            b.s0[d] = src_start ? src_start[k] : 0;
            b.d0[d] = dst_start ? dst_start[k] : 0;
            if (b.ext[d] < 0 || b.s0[d] < 0 || b.d0[d] < 0 || b.s0[d] + b.ext[d] > b.ss[d] ||
                b.d0[d] + b.ext[d] > b.ds[d])
                return fail(DECON_ERR_VALUE, "window outside the array on axis %d", k);
        }
        n *= b.ds[d];
    }
    if (n == 0) return DECON_OK;
    k_window_copy<<<grid1d(n, 256), 256, 0, as_stream(stream)>>>(src, dst, b, n);
    DK_LAUNCHED();
    return DECON_OK;
}

int decon_band_widths(int64_t n_large, int64_t n_small, int* w_fwd, int* w_adj) {
    if (n_large < 1 || n_small < 1) return fail(DECON_ERR_VALUE, "band sizes must be positive");
    const double s = (double)n_large / (double)n_small;
    if (w_fwd) *w_fwd = (int)std::min<int64_t>(n_large, (int64_t)std::ceil(s) + 2);
    if (w_adj) *w_adj = (int)std::min<int64_t>(n_small, (int64_t)std::ceil(1.0 / s) + 3);
    return DECON_OK;
}

int decon_band_weights(int64_t n_large, int64_t n_small, int32_t* idx_f, float* w_f,
                       int32_t* idx_a, float* w_a) {
    int wf = 0, wa = 0;
    DK_TRY(decon_band_widths(n_large, n_small, &wf, &wa));
    const double s = (double)n_large / (double)n_small;
    // large -> small: output cell [i s, (i+1) s) against unit cells [j, j+1)
    for (int64_t i = 0; i < n_small; ++i) {
        int64_t first = (int64_t)std::floor((double)i * s);
        first = std::min<int64_t>(std::max<int64_t>(first, 0), n_large - wf);
        const double lo = (double)i * s, hi = (double)(i + 1) * s;
        for (int k = 0; k < wf; ++k) {
            const int64_t j = first + k;
            const double jd = (double)j;
            if (idx_f) idx_f[i * wf + k] = (int32_t)j;
            if (w_f) w_f[i * wf + k] = (float)std::max(0.0, std::min(hi, jd + 1) - std::max(lo, jd));
        }
    }
    // small -> large (exact transpose derived independently)
    for (int64_t j = 0; j < n_large; ++j) {
        int64_t first = (int64_t)std::floor((double)j / s) - 1;
        first = std::min<int64_t>(std::max<int64_t>(first, 0), n_small - wa);
        const double b = (double)j;
        for (int k = 0; k < wa; ++k) {
            const int64_t i = first + k;
            const double lo = (double)i * s, hi = ((double)i + 1) * s;
            if (idx_a) idx_a[j * wa + k] = (int32_t)i;
            if (w_a) w_a[j * wa + k] = (float)std::max(0.0, std::min(hi, b + 1) - std::max(lo, b));
        }
    }
    return DECON_OK;
}

int decon_banded_axis(const float* in, float* out, int64_t outer, int64_t n_in, int64_t inner,
                      int64_t n_out, const int32_t* idx, const float* w, int width, void* stream) {
    if (!in || !out || !idx || !w) return fail(DECON_ERR_NULL, "null pointer");
    if (outer < 0 || inner < 0 || n_in < 1 || n_out < 1 || width < 1)
        return fail(DECON_ERR_VALUE, "bad banded shape");
    const int64_t n = outer * n_out * inner;
    if (n == 0) return DECON_OK;
    const cudaStream_t st = as_stream(stream);
    if (inner == 1) {
        if (width <= kBandW) {
            // enough CTAs to fill the GPU, each walking many rows
            const int64_t gx = cdiv(n_out, 256);
            const int64_t gy = std::max<int64_t>(1, std::min<int64_t>(outer, cdiv((int64_t)sm_count() * 16, gx)));
            dim3 g((unsigned)gx, (unsigned)gy);
            k_banded_last_rows<<<g, 256, 0, st>>>(in, out, outer, n_in, n_out, idx, w, width);
        } else {
            dim3 g((unsigned)cdiv(n_out, 256), (unsigned)std::min<int64_t>(outer, 65535));
            k_banded_last<<<g, 256, 0, st>>>(in, out, outer, n_in, n_out, idx, w, width);
        }
    } else {
        if (n_out > 65535) return fail(DECON_ERR_UNSUPPORTED, "resampled axis longer than 65535");
        const bool v4 = (inner % 4) == 0 && (reinterpret_cast<uintptr_t>(in) & 15) == 0 &&
                        (reinterpret_cast<uintptr_t>(out) & 15) == 0;
        const int64_t cols = v4 ? inner / 4 : inner;
        const int thr = cols >= 256 ? 256 : (int)round_up(cols, 32);
        dim3 g((unsigned)cdiv(cols, thr), (unsigned)n_out, (unsigned)std::min<int64_t>(outer, 65535));
        if (v4) k_banded_inner4<<<g, thr, 0, st>>>(in, out, outer, n_in, inner, n_out, idx, w, width);
        else k_banded_inner<<<g, thr, 0, st>>>(in, out, outer, n_in, inner, n_out, idx, w, width);
    }
    DK_LAUNCHED();
    return DECON_OK;
}

int decon_hessian3d_forward(const float* x, float* h, const int64_t shape[3], float r, void* stream) {
    if (!x || !h || !shape) return fail(DECON_ERR_NULL, "null pointer");
    W6 w;
    hessian_weights(r, w.w);
    const int64_t n = shape[0] * shape[1] * shape[2];
    if (n <= 0) return DECON_OK;
    const Dims d{shape[0], shape[1], shape[2]};
    const int64_t grid = std::min<int64_t>(TileGeo(d).ntiles, (int64_t)sm_count() * 8);
    if (offsets_fit_u32(d))
        k_hessian_fwd_z<uint32_t><<<(unsigned)std::max<int64_t>(grid, 1), 256, 0, as_stream(stream)>>>(x, h, d, w);
    else
        k_hessian_fwd_z<int64_t><<<(unsigned)std::max<int64_t>(grid, 1), 256, 0, as_stream(stream)>>>(x, h, d, w);
    DK_LAUNCHED();
    return DECON_OK;
}

int decon_hessian3d_adjoint(const float* h, float* x, const int64_t shape[3], float r, void* stream) {
    if (!h || !x || !shape) return fail(DECON_ERR_NULL, "null pointer");
    W6 w;
    hessian_weights(r, w.w);
    const int64_t n = shape[0] * shape[1] * shape[2];
    if (n <= 0) return DECON_OK;
    // the staged tile walk of the fused PDHG kernels (116 vs 227 us for a
    // per-voxel global-memory kernel at 128x256x256, bit-identical)
    return hess_adjoint_tiled(h, x, Dims{shape[0], shape[1], shape[2]}, w, as_stream(stream));
}

int decon_gradient3d_forward(const float* x, float* g, const int64_t shape[3], float r, void* stream) {
    if (!x || !g || !shape) return fail(DECON_ERR_NULL, "null pointer");
    Vol f{x, shape[0], shape[1], shape[2]};
    const int64_t n = shape[0] * shape[1] * shape[2];
    k_gradient_fwd<<<grid1d(n, 256), 256, 0, as_stream(stream)>>>(f, g, r);
    DK_LAUNCHED();
    return DECON_OK;
}

int decon_gradient3d_adjoint(const float* g, float* x, const int64_t shape[3], float r, void* stream) {
    if (!g || !x || !shape) return fail(DECON_ERR_NULL, "null pointer");
    const int64_t n = shape[0] * shape[1] * shape[2];
    k_gradient_adj<<<grid1d(n, 256), 256, 0, as_stream(stream)>>>(g, x, shape[0], shape[1], shape[2], r);
    DK_LAUNCHED();
    return DECON_OK;
}

}  // extern "C"
