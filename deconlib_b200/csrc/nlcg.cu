// Nonlinear conjugate gradients for Poisson maximum likelihood, f = s^2
// (deconlib's nlcg_mlx.py: Schaefer, Schuster & Herz 2001 objective,
// Fletcher-Reeves directions, exact Newton-Raphson step length).
//
// The convolutions and the regulariser run through the operators the caller
// passes; this file holds every other pass of an iteration, each one fused
// elementwise kernel with its FP64 sums:
//
//   k_nlcg_products   d <- r + gamma d (or d as given), s d, d^2
//   k_nlcg_gram       six inner products of C f, C(s d), C(d^2)
//   k_nlcg_newton     one Newton-Raphson refinement of the step length: the
//                     data sums of phi'(lam), phi''(lam); the last CTA adds
//                     the regulariser's terms (polynomials in lam of the Gram
//                     entries) and updates lam on the device
//   k_nlcg_accept_d   model m(lam) = Kss + 2 lam K(sd) + lam^2 K(dd) + b, the
//                     gradient weight 1 - g / m, objective and I-divergence sums
//   k_nlcg_accept_o   s + lam d and its square
//   k_nlcg_gradient   r = -(2 s K^T w + 4 beta s C^T C f), |r|^2, the
//                     I-divergence between successive f and sum f
//
// Element-wise passes move four values per thread and array with float4
// loads and stores when the arrays are 16-byte aligned (ew4).  Every
// reduction is deterministic: each CTA writes its FP64 partials, and
// the last CTA to finish (a ticket counter, no waiting) folds them in block
// order.  The Newton loop runs on the device (lam never leaves HBM), so an
// iteration needs one host read, after the speculative gradient.
#include <cfloat>
#include <initializer_list>

#include "conv_impl.cuh"
#include "zwalk.cuh"

namespace dk {

constexpr int kNlThreads = 256;
constexpr int kNlMaxBlocks = 1184;  // 148 SMs x 8
constexpr int kNlSlots = 6;

struct NlcgDev {
    double lam;
    int done;        // Newton stopped: degenerate curvature or non-finite step
    int newton_run;  // refinements performed
    double gram[6];  // <A,A> <A,B> <A,C> <B,B> <B,C> <C,C> for A = Cf, B = C(sd), C = C(dd)
    double data[3];  // sum m, sum g ln max(m, eps), sum of Poisson I-divergence terms
    double reg[1];   // sum (C f)^2
    double obj[3];   // sum r^2, I-divergence(f_prev, f), sum f
    double quad[2];  // helper sums
    double nt[3];    // Newton data sums (last refinement)
    unsigned ticket;
};

__device__ __forceinline__ int64_t gstride() { return (int64_t)gridDim.x * blockDim.x; }
__device__ __forceinline__ int64_t gtid() { return (int64_t)blockIdx.x * blockDim.x + threadIdx.x; }

// Block sums of v[0..NS) into partials; the last CTA folds them (block order,
// FP64) into out[0..NS) and re-arms the ticket.  Returns true in the last CTA.
template <int NS>
__device__ bool fold_last(double (&v)[NS], double* __restrict__ part, unsigned* ticket,
                          double* out) {
    __shared__ bool last;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        const double t = block_sum(v[s]);
        if (threadIdx.x == 0) part[s * gridDim.x + blockIdx.x] = t;
    }
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int G = (int)gridDim.x;
    for (int s = warp; s < NS; s += blockDim.x >> 5) {
        // eight of the lane's partials in flight at a time, summed in block order
        double acc = 0.0;
        for (int b0 = lane; b0 < G; b0 += 32 * 8) {
            double q[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int b = b0 + 32 * u;
                q[u] = b < G ? __ldcg(&part[s * G + b]) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) acc += q[u];
        }
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if (lane == 0) out[s] = acc;
    }
    __syncthreads();
    if (threadIdx.x == 0) *ticket = 0;
    return true;
}

// Element-wise loop over n values of NI inputs and NO outputs: groups of four
// with float4 loads and stores when `vec` (every pointer 16-byte aligned),
// then the remainder one by one.  f(in[NI], out[NO]) handles one element;
// a null input reads 0, a null output is not stored.
template <int NI, int NO, class F>
__device__ __forceinline__ void ew4(int64_t n, const float* const (&in)[NI], float* const (&out)[NO],
                                    bool vec, F&& f) {
    const int64_t ng = vec ? n / 4 : 0;
    for (int64_t gi = gtid(); gi < ng; gi += gstride()) {
        float4 a[NI];
#pragma unroll
        for (int k = 0; k < NI; ++k)
            a[k] = in[k] ? __ldg(reinterpret_cast<const float4*>(in[k]) + gi) : make_float4(0.f, 0.f, 0.f, 0.f);
        float o[NO][4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            float x[NI], y[NO];
#pragma unroll
            for (int k = 0; k < NI; ++k) x[k] = e == 0 ? a[k].x : e == 1 ? a[k].y : e == 2 ? a[k].z : a[k].w;
            f(x, y);
#pragma unroll
            for (int k = 0; k < NO; ++k) o[k][e] = y[k];
        }
#pragma unroll
        for (int k = 0; k < NO; ++k)
            if (out[k]) reinterpret_cast<float4*>(out[k])[gi] = make_float4(o[k][0], o[k][1], o[k][2], o[k][3]);
    }
    for (int64_t i = 4 * ng + gtid(); i < n; i += gstride()) {
        float x[NI], y[NO];
#pragma unroll
        for (int k = 0; k < NI; ++k) x[k] = in[k] ? in[k][i] : 0.f;
        f(x, y);
#pragma unroll
        for (int k = 0; k < NO; ++k)
            if (out[k]) out[k][i] = y[k];
    }
}

// f0 = max(x, 1e-6), s = sqrt(f0), f = s s; or (from_s) f = s s alone.
__global__ void k_nlcg_init(const float* __restrict__ x, float* __restrict__ s, float* __restrict__ f,
                            int64_t n, int from_s, int vec) {
    const float* in[1] = {x};
    float* out[2] = {from_s ? nullptr : s, f};
    ew4(n, in, out, vec, [&](const float* v, float* o) {
        const float sv = from_s ? v[0] : sqrtf(fmaxf(v[0], 1e-6f));
        o[0] = sv;
        o[1] = sv * sv;
    });
}

// Data-space terms of a model m: w = 1 - g / max(m, eps); sums of m,
// g ln max(m, eps) and the Poisson I-divergence (rl_mlx.py:58-80, eps 1e-6).
__device__ __forceinline__ void model_terms(float m, float g, float eps, float& w, double (&v)[3]) {
    const float mm = fmaxf(m, eps);
    w = 1.0f - g / mm;
    v[0] += (double)m;
    v[1] += (double)(g * logf(mm));
    const float gs = fmaxf(g, 1e-6f), ms = fmaxf(m, 1e-6f);
    v[2] += (double)(g * logf(gs / ms) - (g - ms));
}

__global__ void k_nlcg_model(const float* __restrict__ m, const float* __restrict__ g, float eps,
                             float* __restrict__ w, int64_t n, int vec, double* part, NlcgDev* dev) {
    double v[3] = {0.0, 0.0, 0.0};
    const float* in[2] = {m, g};
    float* out[1] = {w};
    ew4(n, in, out, vec, [&](const float* x, float* o) { model_terms(x[0], x[1], eps, o[0], v); });
    fold_last<3>(v, part, &dev->ticket, dev->data);
}

// mode 0: direction d as given; mode 1: d_out = r + gamma d.  sd = s d, dd = d d.
// Arms the Newton state (lam = 0).
__global__ void k_nlcg_products(int mode, float gamma, const float* __restrict__ s,
                                const float* __restrict__ d, const float* __restrict__ r,
                                float* __restrict__ d_out, float* __restrict__ sd,
                                float* __restrict__ dd, int64_t n, int vec, NlcgDev* dev) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        dev->lam = 0.0;
        dev->done = 0;
        dev->newton_run = 0;
    }
    const float* in[3] = {s, d, mode == 1 ? r : nullptr};
    float* out[3] = {mode == 1 ? d_out : nullptr, sd, dd};
    ew4(n, in, out, vec, [&](const float* x, float* o) {
        const float dv = mode == 1 ? x[2] + gamma * x[1] : x[1];
        o[0] = dv;
        o[1] = x[0] * dv;
        o[2] = dv * dv;
    });
}

__global__ void k_nlcg_gram(const float* __restrict__ a, const float* __restrict__ b,
                            const float* __restrict__ c, int64_t n, int vec, double* part, NlcgDev* dev) {
    double v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    const float* in[3] = {a, b, c};
    float* out[1] = {nullptr};
    ew4(n, in, out, vec, [&](const float* q, float*) {
        const double x = q[0], y = q[1], z = q[2];
        v[0] += x * x;
        v[1] += x * y;
        v[2] += x * z;
        v[3] += y * y;
        v[4] += y * z;
        v[5] += z * z;
    });
    fold_last<6>(v, part, &dev->ticket, dev->gram);
}

// One refinement (nlcg_mlx.py:262-291): data sums at the current lam, then
// lam <- lam - phi' / phi'' in the last CTA.
__global__ void k_nlcg_newton(const float* __restrict__ m, const float* __restrict__ ksd,
                              const float* __restrict__ kdd, const float* __restrict__ g, float b,
                              float eps, double beta, int use_reg, int64_t n, int vec, double* part,
                              NlcgDev* dev) {
    if (dev->done) return;  // every CTA reads the same flag: all return or none
    const double lam = dev->lam;
    const float c1 = (float)(2.0 * lam), c2 = (float)(lam * lam), lf = (float)lam;
    double v[3] = {0.0, 0.0, 0.0};
    const float* in[4] = {m, ksd, kdd, g};
    float* out[1] = {nullptr};
    ew4(n, in, out, vec, [&](const float* x, float*) {
        const float kss = x[0] - b, sdv = x[1], ddv = x[2], gv = x[3];
        const float ml = fmaxf(kss + c1 * sdv + c2 * ddv + b, eps);
        const float sl = sdv + lf * ddv;
        const float wl = 1.0f - gv / ml;
        v[0] += (double)(sl * wl);
        v[1] += (double)(ddv * wl);
        v[2] += (double)(gv * (sl * sl) / (ml * ml));
    });
    if (!fold_last<3>(v, part, &dev->ticket, dev->nt)) return;
    if (threadIdx.x != 0) return;
    double d1 = 2.0 * dev->nt[0];
    double d2 = 2.0 * dev->nt[1] + 4.0 * dev->nt[2];
    if (use_reg) {
        // u = A + 2 lam B + lam^2 C, B_lam = B + lam C (regulariser images of
        // f(lam) and of its lam-derivative / 2): the sums are polynomials in lam.
        const double* G = dev->gram;  // AA AB AC BB BC CC
        const double l = lam, l2 = lam * lam, l3 = l2 * lam;
        const double u_b = G[1] + l * (G[2] + 2.0 * G[3]) + 3.0 * l2 * G[4] + l3 * G[5];
        const double b_b = G[3] + 2.0 * l * G[4] + l2 * G[5];
        const double u_c = G[2] + 2.0 * l * G[4] + l2 * G[5];
        d1 += 4.0 * beta * u_b;
        d2 += 8.0 * beta * b_b + 4.0 * beta * u_c;
    }
    dev->newton_run += 1;
    if (!isfinite(d2) || fabs(d2) < (double)eps) {
        dev->done = 1;
        return;
    }
    const double next = lam - d1 / d2;
    dev->lam = next;
    if (!isfinite(next)) dev->done = 1;
}

// The trial point's model and its data terms (nlcg_mlx.py:297-298, 96-111).
__global__ void k_nlcg_accept_d(const float* __restrict__ m, const float* __restrict__ ksd,
                                const float* __restrict__ kdd, const float* __restrict__ g, float b,
                                float eps, float* __restrict__ m_new, float* __restrict__ w_new,
                                int64_t n, int vec, double* part, NlcgDev* dev) {
    const double lam = dev->lam;
    const float c1 = (float)(2.0 * lam), c2 = (float)(lam * lam);
    double v[3] = {0.0, 0.0, 0.0};
    const float* in[4] = {m, ksd, kdd, g};
    float* out[2] = {m_new, w_new};
    ew4(n, in, out, vec, [&](const float* x, float* o) {
        const float kss = x[0] - b;
        const float mn = kss + c1 * x[1] + c2 * x[2] + b;
        o[0] = mn;
        model_terms(mn, x[3], eps, o[1], v);
    });
    fold_last<3>(v, part, &dev->ticket, dev->data);
}

__global__ void k_nlcg_accept_o(const float* __restrict__ s, const float* __restrict__ d,
                                float* __restrict__ s_new, float* __restrict__ f_new, int64_t n, int vec,
                                const NlcgDev* dev) {
    const float lf = (float)dev->lam;
    const float* in[2] = {s, d};
    float* out[2] = {s_new, f_new};
    ew4(n, in, out, vec, [&](const float* x, float* o) {
        const float sn = x[0] + lf * x[1];
        o[0] = sn;
        o[1] = sn * sn;
    });
}

__global__ void k_nlcg_energy(const float* __restrict__ a, int64_t n, int vec, double* part, NlcgDev* dev) {
    double v[1] = {0.0};
    const float* in[1] = {a};
    float* out[1] = {nullptr};
    ew4(n, in, out, vec, [&](const float* x, float*) {
        const double q = x[0];
        v[0] += q * q;
    });
    fold_last<1>(v, part, &dev->ticket, dev->reg);
}

// r = -(2 s K^T w [+ 4 beta s C^T C f]) (nlcg_mlx.py:105-115), sum r^2 (skipped
// without ktw); with f_prev: the I-divergence of f against f_prev
// (nlcg_mlx.py:303-323); sum f.
__global__ void k_nlcg_gradient(const float* __restrict__ s, const float* __restrict__ f,
                                const float* __restrict__ f_prev, const float* __restrict__ ktw,
                                const float* __restrict__ ctcf, float c4b, float eps,
                                float* __restrict__ r, int64_t n, int vec, double* part, NlcgDev* dev) {
    double v[3] = {0.0, 0.0, 0.0};
    const bool has_g = ktw != nullptr, has_c = ctcf != nullptr, has_p = f_prev != nullptr;
    const float* in[5] = {has_g ? s : nullptr, f, f_prev, ktw, ctcf};
    float* out[1] = {has_g ? r : nullptr};
    ew4(n, in, out, vec, [&](const float* x, float* o) {
        o[0] = 0.f;
        if (has_g) {
            const float sv = x[0];
            float grad = (2.0f * sv) * x[3];
            if (has_c) grad = grad + (c4b * sv) * x[4];
            const float rv = -grad;
            o[0] = rv;
            v[0] += (double)rv * (double)rv;
        }
        const float fc = x[1];
        if (has_p) {
            const float fp = x[2];
            v[1] += (double)(fp * (logf(fmaxf(fp, eps)) - logf(fmaxf(fc, eps))) - fp + fc);
        }
        v[2] += (double)fc;
    });
    fold_last<3>(v, part, &dev->ticket, dev->obj);
}

// Hessian3D regulariser without materialising its images (the 6-component
// fields C f, C(s d), C(d^2)): their Gram matrix and ||C f||^2 with the
// components evaluated on the fly by the register z-walk (zwalk.cuh), whose
// float operations are the operator's.
struct Fields3 {
    float a, b, c;
};

template <class IDX>
__global__ void __launch_bounds__(256) k_nlcg_hess_gram(const float* __restrict__ f,
                                                        const float* __restrict__ sd,
                                                        const float* __restrict__ dd, Dims d, W6 w,
                                                        double* part, NlcgDev* dev) {
    double v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    hess_zwalk<IDX, 3>(
        d, w, [&](IDX i) { return Fields3{__ldg(f + i), __ldg(sd + i), __ldg(dd + i)}; },
        [](const Fields3& r, int k) { return k == 0 ? r.a : (k == 1 ? r.b : r.c); },
        [&](IDX, const float (*h)[6]) {
            // the six-component products of one voxel in FP32, the sum over
            // voxels in FP64
            float p[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int q = 0; q < 6; ++q) {
                const float x = h[0][q], y = h[1][q], z = h[2][q];
                p[0] = fmaf(x, x, p[0]);
                p[1] = fmaf(x, y, p[1]);
                p[2] = fmaf(x, z, p[2]);
                p[3] = fmaf(y, y, p[3]);
                p[4] = fmaf(y, z, p[4]);
                p[5] = fmaf(z, z, p[5]);
            }
#pragma unroll
            for (int q = 0; q < 6; ++q) v[q] += (double)p[q];
        });
    fold_last<6>(v, part, &dev->ticket, dev->gram);
}

template <class IDX>
__global__ void __launch_bounds__(256) k_nlcg_hess_energy(const float* __restrict__ f, Dims d, W6 w,
                                                          double* part, NlcgDev* dev) {
    double v[1] = {0.0};
    hess_zwalk<IDX, 1>(
        d, w, [&](IDX i) { return __ldg(f + i); }, [](const float& r, int) { return r; },
        [&](IDX, const float (*h)[6]) {
            float p = 0.f;
#pragma unroll
            for (int q = 0; q < 6; ++q) p = fmaf(h[0][q], h[0][q], p);
            v[0] += (double)p;
        });
    fold_last<1>(v, part, &dev->ticket, dev->reg);
}

// Quadratic-form helper sums (nlcg_mlx.py:181-193):
// quad[0] = sum (g / max(m m, eps)) K(sd)^2, quad[1] = sum a d^2.
__global__ void k_nlcg_quad(const float* __restrict__ g, const float* __restrict__ m,
                            const float* __restrict__ ksd, int64_t nd, const float* __restrict__ a,
                            const float* __restrict__ d, int64_t no, float eps, double* part,
                            NlcgDev* dev) {
    double v[2] = {0.0, 0.0};
    for (int64_t i = gtid(); i < nd; i += gstride()) {
        const float mv = m[i], kv = ksd[i];
        v[0] += (double)((g[i] / fmaxf(mv * mv, eps)) * (kv * kv));
    }
    for (int64_t i = gtid(); i < no; i += gstride()) {
        const float dv = d[i];
        v[1] += (double)(a[i] * (dv * dv));
    }
    fold_last<2>(v, part, &dev->ticket, dev->quad);
}

static int nl_blocks(int64_t n) {
    return (int)std::max<int64_t>(1, std::min<int64_t>(kNlMaxBlocks, cdiv(n, (int64_t)kNlThreads * 4)));
}

// 1 when every non-null pointer is 16-byte aligned (float4 path of ew4).
static int al16(std::initializer_list<const void*> ps) {
    for (const void* p : ps)
        if (p && (reinterpret_cast<uintptr_t>(p) & 15) != 0) return 0;
    return 1;
}

}  // namespace dk

using namespace dk;

struct decon_nlcg {
    NlcgDev* dev = nullptr;
    double* part = nullptr;
    NlcgDev* host = nullptr;  // pinned mirror for decon_nlcg_read
};

static int nl_free(decon_nlcg* h) {
    if (!h) return DECON_OK;
    cudaFree(h->dev);
    cudaFree(h->part);
    cudaFreeHost(h->host);
    delete h;
    return DECON_OK;
}

extern "C" {

int decon_nlcg_create(decon_nlcg** out) {
    if (!out) return fail(DECON_ERR_NULL, "null pointer");
    *out = nullptr;
    decon_nlcg* h = new decon_nlcg();
    if (cudaMalloc(&h->dev, sizeof(NlcgDev)) != cudaSuccess ||
        cudaMalloc(&h->part, sizeof(double) * kNlSlots * kNlMaxBlocks) != cudaSuccess ||
        cudaMallocHost(&h->host, sizeof(NlcgDev)) != cudaSuccess) {
        cudaGetLastError();
        nl_free(h);
        return fail(DECON_ERR_OOM, "decon_nlcg_create: allocation failed");
    }
    if (memset_blocking(h->dev, 0, sizeof(NlcgDev)) != DECON_OK) {
        nl_free(h);
        return fail(DECON_ERR_CUDA, "decon_nlcg_create: memset failed");
    }
    *out = h;
    return DECON_OK;
}

int decon_nlcg_destroy(decon_nlcg* h) { return nl_free(h); }

int decon_nlcg_init(const float* x, float* s, float* f, int64_t n, int from_s, void* stream) {
    if (!x || !f || (!from_s && !s)) return fail(DECON_ERR_NULL, "null pointer");
    if (n <= 0) return DECON_OK;
    k_nlcg_init<<<nl_blocks(n), kNlThreads, 0, as_stream(stream)>>>(x, s, f, n, from_s, al16({x, s, f}));
    DK_LAUNCHED();
    return DECON_OK;
}

int decon_nlcg_model(decon_nlcg* h, const float* m, const float* g, float eps, float* w, int64_t n,
                     void* stream) {
    if (!h || !m || !g) return fail(DECON_ERR_NULL, "null pointer");
    if (n <= 0) return fail(DECON_ERR_VALUE, "decon_nlcg_model: empty data");
    k_nlcg_model<<<nl_blocks(n), kNlThreads, 0, as_stream(stream)>>>(m, g, eps, w, n, al16({m, g, w}),
                                                                     h->part, h->dev);
    DK_LAUNCHED();
    return DECON_OK;
}

int decon_nlcg_products(decon_nlcg* h, int mode, float gamma, const float* s, const float* d,
                        const float* r, float* d_out, float* sd, float* dd, int64_t n, void* stream) {
    if (!h || !s || !d || !sd || !dd || (mode == 1 && (!r || !d_out)))
        return fail(DECON_ERR_NULL, "null pointer");
    if (mode != 0 && mode != 1) return fail(DECON_ERR_VALUE, "decon_nlcg_products: mode must be 0 or 1");
    if (n <= 0) return fail(DECON_ERR_VALUE, "decon_nlcg_products: empty object");
    const int vec = al16({s, d, mode == 1 ? r : nullptr, mode == 1 ? d_out : nullptr, sd, dd});
    k_nlcg_products<<<nl_blocks(n), kNlThreads, 0, as_stream(stream)>>>(mode, gamma, s, d, r, d_out, sd,
                                                                        dd, n, vec, h->dev);
    DK_LAUNCHED();
    return DECON_OK;
}

int decon_nlcg_gram(decon_nlcg* h, const float* a, const float* b, const float* c, int64_t n,
                    void* stream) {
    if (!h || !a || !b || !c) return fail(DECON_ERR_NULL, "null pointer");
    if (n <= 0) return fail(DECON_ERR_VALUE, "decon_nlcg_gram: empty");
    k_nlcg_gram<<<nl_blocks(n), kNlThreads, 0, as_stream(stream)>>>(a, b, c, n, al16({a, b, c}), h->part,
                                                                    h->dev);
    DK_LAUNCHED();
    return DECON_OK;
}

int decon_nlcg_newton(decon_nlcg* h, const float* m, const float* ksd, const float* kdd, const float* g,
                      float background, float eps, double beta, int use_reg, int newton_iters,
                      int64_t n, void* stream) {
    if (!h || !m || !ksd || !kdd || !g) return fail(DECON_ERR_NULL, "null pointer");
    if (n <= 0) return fail(DECON_ERR_VALUE, "decon_nlcg_newton: empty data");
    const cudaStream_t st = as_stream(stream);
    for (int it = 0; it < newton_iters; ++it) {
        k_nlcg_newton<<<nl_blocks(n), kNlThreads, 0, st>>>(m, ksd, kdd, g, background, eps, beta, use_reg,
                                                          n, al16({m, ksd, kdd, g}), h->part, h->dev);
        DK_LAUNCHED();
    }
    return DECON_OK;
}

int decon_nlcg_accept(decon_nlcg* h, const float* m, const float* ksd, const float* kdd, const float* g,
                      float background, float eps, float* m_new, float* w_new, int64_t nd,
                      const float* s, const float* d, float* s_new, float* f_new, int64_t no,
                      void* stream) {
    if (!h || !m || !ksd || !kdd || !g || !m_new) return fail(DECON_ERR_NULL, "null pointer");
    if (nd <= 0) return fail(DECON_ERR_VALUE, "decon_nlcg_accept: empty data");
    const cudaStream_t st = as_stream(stream);
    k_nlcg_accept_d<<<nl_blocks(nd), kNlThreads, 0, st>>>(m, ksd, kdd, g, background, eps, m_new, w_new,
                                                         nd, al16({m, ksd, kdd, g, m_new, w_new}), h->part,
                                                         h->dev);
    DK_LAUNCHED();
    if (s) {
        if (!d || !s_new || !f_new) return fail(DECON_ERR_NULL, "null pointer");
        k_nlcg_accept_o<<<nl_blocks(no), kNlThreads, 0, st>>>(s, d, s_new, f_new, no,
                                                             al16({s, d, s_new, f_new}), h->dev);
        DK_LAUNCHED();
    }
    return DECON_OK;
}

int decon_nlcg_energy(decon_nlcg* h, const float* a, int64_t n, void* stream) {
    if (!h || !a) return fail(DECON_ERR_NULL, "null pointer");
    if (n <= 0) return fail(DECON_ERR_VALUE, "decon_nlcg_energy: empty");
    k_nlcg_energy<<<nl_blocks(n), kNlThreads, 0, as_stream(stream)>>>(a, n, al16({a}), h->part, h->dev);
    DK_LAUNCHED();
    return DECON_OK;
}

int decon_nlcg_gradient(decon_nlcg* h, const float* s, const float* f, const float* f_prev,
                        const float* ktw, const float* ctcf, float c4b, float eps, float* r, int64_t n,
                        void* stream) {
    if (!h || !f || (ktw && (!s || !r))) return fail(DECON_ERR_NULL, "null pointer");
    if (n <= 0) return fail(DECON_ERR_VALUE, "decon_nlcg_gradient: empty object");
    const int vec = al16({ktw ? s : nullptr, f, f_prev, ktw, ctcf, ktw ? r : nullptr});
    k_nlcg_gradient<<<nl_blocks(n), kNlThreads, 0, as_stream(stream)>>>(s, f, f_prev, ktw, ctcf, c4b, eps,
                                                                       r, n, vec, h->part, h->dev);
    DK_LAUNCHED();
    return DECON_OK;
}

static int hess_grid(const Dims& d, const void* fn) {
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, 256, 0) != cudaSuccess) {
        cudaGetLastError();
        occ = 1;
    }
    const int64_t cap = std::min<int64_t>(kNlMaxBlocks, (int64_t)sm_count() * std::max(occ, 1));
    return (int)std::max<int64_t>(1, std::min<int64_t>(TileGeo(d).ntiles, cap));
}

int decon_nlcg_hess_gram(decon_nlcg* h, const float* f, const float* sd, const float* dd,
                         const int64_t shape[3], float r, void* stream) {
    if (!h || !f || !sd || !dd || !shape) return fail(DECON_ERR_NULL, "null pointer");
    if (shape[0] < 1 || shape[1] < 1 || shape[2] < 1) return fail(DECON_ERR_VALUE, "decon_nlcg_hess_gram: empty");
    const Dims d{shape[0], shape[1], shape[2]};
    W6 w;
    hessian_weights(r, w.w);
    if (offsets_fit_u32(d))
        k_nlcg_hess_gram<uint32_t><<<hess_grid(d, (const void*)k_nlcg_hess_gram<uint32_t>), 256, 0, as_stream(stream)>>>(
            f, sd, dd, d, w, h->part, h->dev);
    else
        k_nlcg_hess_gram<int64_t><<<hess_grid(d, (const void*)k_nlcg_hess_gram<int64_t>), 256, 0, as_stream(stream)>>>(
            f, sd, dd, d, w, h->part, h->dev);
    DK_LAUNCHED();
    return DECON_OK;
}

int decon_nlcg_hess_energy(decon_nlcg* h, const float* f, const int64_t shape[3], float r, void* stream) {
    if (!h || !f || !shape) return fail(DECON_ERR_NULL, "null pointer");
    if (shape[0] < 1 || shape[1] < 1 || shape[2] < 1) return fail(DECON_ERR_VALUE, "decon_nlcg_hess_energy: empty");
    const Dims d{shape[0], shape[1], shape[2]};
    W6 w;
    hessian_weights(r, w.w);
    if (offsets_fit_u32(d))
        k_nlcg_hess_energy<uint32_t><<<hess_grid(d, (const void*)k_nlcg_hess_energy<uint32_t>), 256, 0,
                                       as_stream(stream)>>>(f, d, w, h->part, h->dev);
    else
        k_nlcg_hess_energy<int64_t><<<hess_grid(d, (const void*)k_nlcg_hess_energy<int64_t>), 256, 0,
                                      as_stream(stream)>>>(f, d, w, h->part, h->dev);
    DK_LAUNCHED();
    return DECON_OK;
}

int decon_nlcg_quad(decon_nlcg* h, const float* g, const float* m, const float* ksd, int64_t nd,
                    const float* a, const float* d, int64_t no, float eps, void* stream) {
    if (!h || !g || !m || !ksd || !a || !d) return fail(DECON_ERR_NULL, "null pointer");
    if (nd <= 0 || no <= 0) return fail(DECON_ERR_VALUE, "decon_nlcg_quad: empty");
    const int64_t big = std::max(nd, no);
    k_nlcg_quad<<<nl_blocks(big), kNlThreads, 0, as_stream(stream)>>>(g, m, ksd, nd, a, d, no, eps,
                                                                     h->part, h->dev);
    DK_LAUNCHED();
    return DECON_OK;
}

// Synchronises `stream` and returns the scalars: out[0] lam, [1] Newton
// stopped (0/1), [2] refinements run, [3..5] data sums (sum m,
// sum g ln max(m, eps), sum I-divergence terms), [6] regulariser energy,
// [7..9] sum r^2, I-divergence between iterates, sum f, [10..11] quadratic-form
// sums, [12..17] Gram entries.
int decon_nlcg_read(decon_nlcg* h, double* out, void* stream) {
    if (!h || !out) return fail(DECON_ERR_NULL, "null pointer");
    const cudaStream_t st = as_stream(stream);
    DK_CUDA(cudaMemcpyAsync(h->host, h->dev, sizeof(NlcgDev), cudaMemcpyDeviceToHost, st));
    DK_CUDA(cudaStreamSynchronize(st));
    const NlcgDev& v = *h->host;
    out[0] = v.lam;
    out[1] = v.done;
    out[2] = v.newton_run;
    for (int i = 0; i < 3; ++i) out[3 + i] = v.data[i];
    out[6] = v.reg[0];
    for (int i = 0; i < 3; ++i) out[7 + i] = v.obj[i];
    out[10] = v.quad[0];
    out[11] = v.quad[1];
    for (int i = 0; i < 6; ++i) out[12 + i] = v.gram[i];
    return DECON_OK;
}

}  // extern "C"
