// Solver kernels: adaptive PDHG (Malitsky-Pock) with device-resident step
// sizes, and the element-wise Richardson-Lucy steps for composed operators.
//
// PDHG (deconvolution/pdhg_mlx.py:717-900 / :1066-1221) keeps tau, sigma,
// theta, the convergence counter and the histories in device memory.  Every
// kernel that changes solver state reads them from there and returns at once
// when the stop flag is set, so a host can queue many iterations without
// synchronising; the FP64 reductions (||dx||^2, ||x||^2, ||dKx||^2, losses)
// are folded in fixed order by the one-CTA step kernel.
#include <cfloat>
#include <cstddef>
#include <map>
#include <mutex>

#include "conv_impl.cuh"
#include "solvers.cuh"
#include "stencil.cuh"
#include "pdhg_tiled.cuh"

namespace dk {

constexpr int kSlotDx2 = 0, kSlotXc2 = 1, kSlotXn2 = 2, kSlotDA2 = 3, kSlotDL2 = 4,
              kSlotData = 5, kSlotReg = 6;

// The objective of iteration kk is recorded unless the solve stopped before
// it or broke on convergence at it (pdhg_mlx.py:812-833 break before :860).
__device__ __forceinline__ bool loss_active(const PdhgDev* s, int kk) {
    return kk < s->final_iter && !(s->converged && kk == s->final_iter - 1);
}

__device__ __forceinline__ void put_partial(PdhgDev* s, int slot, double v) {
    const double b = block_sum(v);
    if (threadIdx.x == 0) s->partials[slot * kPdhgGrid + blockIdx.x] = b;
}

// ---- data-term dual: y1 = prox(y1 + sigma * A xbar) (pdhg_mlx.py:723-728) ----
// A xbar = (1 + theta) A x_cur - theta A x_prev (linearity of A).
template <int LOSS>
__global__ void __launch_bounds__(256) k_dual_data(PdhgDev* s, float* __restrict__ y1,
                                                   const float* __restrict__ axc,
                                                   const float* __restrict__ axp,
                                                   const float* __restrict__ data, float bg,
                                                   int64_t m) {
    if (s->stop) return;
    const float sg = (float)s->sigma, th = (float)s->theta;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float a = axc[i];
        const float axbar = xbar_of(a, axp[i], th);
        const float arg = dual_arg(y1[i], sg, axbar);
        const float d = data[i];
        float out;
        if constexpr (LOSS == 0) {
            // prox_poisson_dual (pdhg_mlx.py:145-166)
            const float c = 1.f - arg - sg * bg;
            const float ds = fmaxf(d, 0.f);
            const float disc = c * c + 4.f * sg * ds;
            float z = (2.f * sg * ds) / (sqrtf(disc) - c + 1e-12f);
            z = ds < 1e-6f ? fmaxf(c, 1e-6f) : z;
            z = fmaxf(z, 1e-6f);
            out = 1.f - z;
        } else {
            // prox_gaussian_dual (pdhg_mlx.py:189)
            out = (arg - sg * (d - bg)) / (1.f + sg);
        }
        y1[i] = out;
    }
}

// ---- regulariser dual: y2 = proj(y2 + sigma * L xbar) (pdhg_mlx.py:732-734) ----
template <int NORM>
__global__ void __launch_bounds__(256) k_dual_reg(PdhgDev* s, float* __restrict__ y2,
                                                  const float* __restrict__ lxbar, float alpha,
                                                  int ncomp, int64_t n) {
    if (s->stop) return;
    const float sg = (float)s->sigma;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        if constexpr (NORM == 0) {
            // prox_l1_dual: clip(y, -alpha, alpha)
            for (int c = 0; c < ncomp; ++c) {
                const int64_t j = (int64_t)c * n + i;
                y2[j] = fminf(fmaxf(dual_arg(y2[j], sg, lxbar[j]), -alpha), alpha);
            }
        } else {
            // prox_l1_2_dual: y / max(sqrt(sum_c y^2 + 1e-12) / alpha, 1)
            float v[8];
            float ss = 0.f;
            for (int c = 0; c < ncomp; ++c) {
                const int64_t j = (int64_t)c * n + i;
                v[c] = dual_arg(y2[j], sg, lxbar[j]);
                ss += v[c] * v[c];
            }
            const float sc = fmaxf(sqrtf(ss + 1e-12f) / alpha, 1.f);
            for (int c = 0; c < ncomp; ++c) y2[(int64_t)c * n + i] = v[c] / sc;
        }
    }
}

// xbar = x_cur + theta (x_cur - x_prev) (pdhg_mlx.py:841)
__global__ void __launch_bounds__(256) k_xbar(PdhgDev* s, const float* __restrict__ xc,
                                              const float* __restrict__ xp, float* __restrict__ xb,
                                              int64_t n) {
    if (s->stop) return;
    const float th = (float)s->theta;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float a = xc[i];
        xb[i] = xbar_of(a, xp[i], th);
    }
}

// x_new = max(0, x - tau (A^T y1 + L^T y2)) and the FP64 sums
// ||x_new - x||^2, ||x||^2, ||x_new||^2 (pdhg_mlx.py:741-750, 805-806).
__global__ void __launch_bounds__(256) k_primal(PdhgDev* s, const float* __restrict__ xc,
                                                const float* __restrict__ aty,
                                                const float* __restrict__ lty,
                                                float* __restrict__ xn, int64_t n) {
    if (s->stop) return;
    const float tau = (float)s->tau;
    double dx2 = 0.0, xc2 = 0.0, xn2 = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float a = xc[i];
        const float g = __fadd_rn(aty[i], lty ? lty[i] : 0.f);
        const float v = primal_of(a, tau, g);
        xn[i] = v;
        const float d = v - a;
        dx2 += (double)d * d;
        xc2 += (double)a * a;
        xn2 += (double)v * v;
    }
    put_partial(s, kSlotDx2, dx2);
    put_partial(s, kSlotXc2, xc2);
    put_partial(s, kSlotXn2, xn2);
}

// sum (a - b)^2 into a slot (||A x_new - A x||^2, pdhg_mlx.py:756-759)
__global__ void __launch_bounds__(256) k_diffsq_slot(PdhgDev* s, const float* __restrict__ a,
                                                     const float* __restrict__ b, int64_t n,
                                                     int slot) {
    if (s->stop) return;
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double d = (double)a[i] - (b ? (double)b[i] : 0.0);
        acc += d * d;
    }
    put_partial(s, slot, acc);
}

// d = a - b (the argument of L (x_new - x))
__global__ void __launch_bounds__(256) k_sub(PdhgDev* s, const float* __restrict__ a,
                                             const float* __restrict__ b, float* __restrict__ d,
                                             int64_t n) {
    if (s->stop) return;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        d[i] = a[i] - b[i];
}

// Loss terms at eval_interval (pdhg_mlx.py:860-881): data part over M.
template <int LOSS>
__global__ void __launch_bounds__(256) k_loss_data(PdhgDev* s, const float* __restrict__ ax,
                                                   const float* __restrict__ data, float bg,
                                                   int64_t m, int kk) {
    if (!loss_active(s, kk)) return;
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float fm = ax[i] + bg;
        const float d = data[i];
        if constexpr (LOSS == 0) {
            const float fms = fmaxf(fm, 1e-6f);
            acc += (double)(d * logf((d + 1e-6f) / fms) - (d - fm));
        } else {
            const float r = d - fm;
            acc += 0.5 * (double)(r * r);
        }
    }
    put_partial(s, kSlotData, acc);
}

// Regulariser part: alpha * sum |Lx| (L1) or alpha * sum sqrt(sum_c (Lx)^2 + 1e-12).
template <int NORM>
__global__ void __launch_bounds__(256) k_loss_reg(PdhgDev* s, const float* __restrict__ lx,
                                                  int ncomp, int64_t n, int kk) {
    if (!loss_active(s, kk)) return;
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        if constexpr (NORM == 0) {
            for (int c = 0; c < ncomp; ++c) acc += fabs((double)lx[(int64_t)c * n + i]);
        } else {
            float ss = 0.f;
            for (int c = 0; c < ncomp; ++c) {
                const float v = lx[(int64_t)c * n + i];
                ss += v * v;
            }
            acc += (double)sqrtf(ss + 1e-12f);
        }
    }
    put_partial(s, kSlotReg, acc);
}

__device__ double fold_slot(const PdhgDev* s, int slot) {
    __shared__ double red[32];
    double v = 0.0;
    for (int i = threadIdx.x; i < kPdhgGrid; i += blockDim.x) v += s->partials[slot * kPdhgGrid + i];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    return t;  // valid in thread 0
}

// The Malitsky-Pock scalar step (pdhg_mlx.py:749-857) in FP64, one CTA.
__global__ void __launch_bounds__(256) k_step(PdhgDev* s) {
    if (s->stop) return;
    // the five FP64 sums folded at once, one warp per slot (fixed order)
    __shared__ double red[5];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp < 5) {
        const int slot = warp == 0 ? kSlotDx2 : warp == 1 ? kSlotXc2 : warp == 2 ? kSlotXn2
                       : warp == 3 ? kSlotDA2 : kSlotDL2;
        const double* p = s->partials + slot * kPdhgGrid;
        // all of a lane's partials loaded at once, then summed in index order
        // (the same sums as a sequential loop, without 19 dependent loads)
        constexpr int kPer = (kPdhgGrid + 31) / 32;
        double q[kPer];
#pragma unroll
        for (int u = 0; u < kPer; ++u) {
            const int i = lane + 32 * u;
            q[u] = i < kPdhgGrid ? p[i] : 0.0;
        }
        double v = 0.0;
#pragma unroll
        for (int u = 0; u < kPer; ++u) v += q[u];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp] = v;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    const double dx2 = red[0], xc2 = red[1], xn2 = red[2], dA2 = red[3], dL2 = red[4];
    const int k = s->k;
    const double tau = s->tau, sigma = s->sigma, theta = s->theta, ss = s->step_scale;
    const double dK2 = dA2 + dL2;
    const double ratio = dx2 / (2.0 * sigma * fmax(dK2, 1e-12));
    const double tau_c = fmin(sqrt(1.0 + theta) * tau, s->delta * sqrt(ratio));
    double tau_n = (tau_c * sigma * dK2 > s->delta * dx2) ? s->eta * tau_c : tau_c;
    tau_n = fmax(tau_n, ss * 1e-4);
    const double theta_n = tau_n / tau;
    double sigma_n = sigma / fmax(theta_n, 0.1);
    sigma_n = fmin(fmax(sigma_n, ss * 1e-4), ss * 1e4);
    const double rel = sqrt(dx2 / (fmax(xc2, xn2) + 1e-12));
    s->rel_hist[k] = rel;
    s->tau_hist[k] = tau_n;
    s->sigma_hist[k] = sigma_n;
    s->last_dx2 = dx2;
    s->last_dK2 = dK2;
    if (k >= s->min_iter) {
        if (rel < s->tol) {
            s->count += 1;
            if (s->count >= s->patience) {
                s->converged = 1;
                s->final_iter = k + 1;
                s->stop = 1;
                s->k = k + 1;
                return;
            }
        } else {
            s->count = 0;
        }
    }
    s->tau = tau_n;
    s->sigma = sigma_n;
    s->theta = theta_n;
    s->k = k + 1;
    if (s->k >= s->num_iter) {
        s->final_iter = s->num_iter;
        s->stop = 1;
    }
}

// Records alpha-weighted loss for iteration k-1 (called after k_step).
__global__ void k_record_loss(PdhgDev* s, double alpha, int kk) {
    if (!loss_active(s, kk)) return;
    const double dl = fold_slot(s, kSlotData);
    const double rl = fold_slot(s, kSlotReg);
    if (threadIdx.x == 0) s->loss_hist[kk] = dl + alpha * rl;
}

// ---- fused Hessian3D PDHG kernels --------------------------------------------
// The regulariser half of the iteration without materialising L x_bar, L^T y2
// or L (x_new - x): the Hessian is evaluated on the fly from the fields below
// (values identical to the stand-alone operator, the same float32 ops).

struct XbarField {  // x_bar = x + theta (x - x_prev)
    const float* xc;
    const float* xp;
    float th;
    int64_t ny, nx;
    __device__ __forceinline__ float operator()(int64_t z, int64_t y, int64_t x) const {
        const int64_t i = (z * ny + y) * nx + x;
        const float a = __ldg(xc + i);
        return xbar_of(a, __ldg(xp + i), th);
    }
};

struct DiffField {  // x_new - x
    const float* a;
    const float* b;
    int64_t ny, nx;
    __device__ __forceinline__ float operator()(int64_t z, int64_t y, int64_t x) const {
        const int64_t i = (z * ny + y) * nx + x;
        return __ldg(a + i) - __ldg(b + i);
    }
};

struct PlainField {
    const float* p;
    int64_t ny, nx;
    __device__ __forceinline__ float operator()(int64_t z, int64_t y, int64_t x) const {
        return __ldg(p + (z * ny + y) * nx + x);
    }
};

// y2 = proj(y2 + sigma H x_bar) (pdhg_mlx.py:732-734 with x_bar of :841).
template <int NORM>
__global__ void __launch_bounds__(256) k_hess_dual(PdhgDev* s, float* __restrict__ y2,
                                                   const float* __restrict__ xc,
                                                   const float* __restrict__ xp, Dims d, W6 w,
                                                   float alpha) {
    if (s->stop) return;
    const float sg = (float)s->sigma;
    const XbarField f{xc, xp, (float)s->theta, d.ny, d.nx};
    const int64_t n = d.nz * d.ny * d.nx;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t x = i % d.nx, t = i / d.nx, y = t % d.ny, z = t / d.ny;
        float h[6];
        hess6(f, z, y, x, d, w.w, h);
        if constexpr (NORM == 0) {
#pragma unroll
            for (int c = 0; c < 6; ++c) {
                const int64_t j = c * n + i;
                y2[j] = fminf(fmaxf(dual_arg(y2[j], sg, h[c]), -alpha), alpha);
            }
        } else {
            float v[6];
            float ss = 0.f;
#pragma unroll
            for (int c = 0; c < 6; ++c) {
                v[c] = dual_arg(y2[c * n + i], sg, h[c]);
                ss += v[c] * v[c];
            }
            const float sc = fmaxf(sqrtf(ss + 1e-12f) / alpha, 1.f);
#pragma unroll
            for (int c = 0; c < 6; ++c) y2[c * n + i] = v[c] / sc;
        }
    }
}

// x_new = max(0, x - tau (A^T y1 + H^T y2)) with the FP64 sums of k_primal.
__global__ void __launch_bounds__(256) k_hess_primal(PdhgDev* s, const float* __restrict__ xc,
                                                     const float* __restrict__ aty,
                                                     const float* __restrict__ y2,
                                                     float* __restrict__ xn, Dims d, W6 w) {
    if (s->stop) return;
    const float tau = (float)s->tau;
    const int64_t n = d.nz * d.ny * d.nx;
    double dx2 = 0.0, xc2 = 0.0, xn2 = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t x = i % d.nx, t = i / d.nx, y = t % d.ny, z = t / d.ny;
        const float a = xc[i];
        const float g = __fadd_rn(aty[i], hess_adj_at(y2, z, y, x, d, w.w));
        const float v = primal_of(a, tau, g);
        xn[i] = v;
        const float dd = v - a;
        dx2 += (double)dd * dd;
        xc2 += (double)a * a;
        xn2 += (double)v * v;
    }
    put_partial(s, kSlotDx2, dx2);
    put_partial(s, kSlotXc2, xc2);
    put_partial(s, kSlotXn2, xn2);
}

// ||A x_new - A x||^2 (slot DA2) and ||H (x_new - x)||^2 (slot DL2).
__global__ void __launch_bounds__(256) k_hess_dk(PdhgDev* s, const float* __restrict__ axn,
                                                 const float* __restrict__ axc, int64_t m,
                                                 const float* __restrict__ xn,
                                                 const float* __restrict__ xc, Dims d, W6 w) {
    if (s->stop) return;
    double a2 = 0.0, l2 = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double dd = (double)axn[i] - (double)axc[i];
        a2 += dd * dd;
    }
    const DiffField f{xn, xc, d.ny, d.nx};
    const int64_t n = d.nz * d.ny * d.nx;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t x = i % d.nx, t = i / d.nx, y = t % d.ny, z = t / d.ny;
        float h[6];
        hess6(f, z, y, x, d, w.w, h);
#pragma unroll
        for (int c = 0; c < 6; ++c) l2 += (double)h[c] * (double)h[c];
    }
    put_partial(s, kSlotDA2, a2);
    put_partial(s, kSlotDL2, l2);
}

// Regulariser part of the objective on H x (pdhg_mlx.py:873-879).
template <int NORM>
__global__ void __launch_bounds__(256) k_hess_regloss(PdhgDev* s, const float* __restrict__ x,
                                                      Dims d, W6 w, int kk) {
    if (!loss_active(s, kk)) return;
    const PlainField f{x, d.ny, d.nx};
    const int64_t n = d.nz * d.ny * d.nx;
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t xx = i % d.nx, t = i / d.nx, y = t % d.ny, z = t / d.ny;
        float h[6];
        hess6(f, z, y, xx, d, w.w, h);
        if constexpr (NORM == 0) {
#pragma unroll
            for (int c = 0; c < 6; ++c) acc += fabs((double)h[c]);
        } else {
            float ss = 0.f;
#pragma unroll
            for (int c = 0; c < 6; ++c) ss += h[c] * h[c];
            acc += (double)sqrtf(ss + 1e-12f);
        }
    }
    put_partial(s, kSlotReg, acc);
}

// ---- RL element-wise steps for composed operators (rl_mlx.py:146-150) -------

__global__ void k_rl_ratio(const float* __restrict__ model, const float* __restrict__ y, float bg,
                           float* __restrict__ ratio, int64_t n, double* __restrict__ partials) {
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float m = model[i] + bg;
        const float yv = y[i];
        if (ratio) ratio[i] = yv / fmaxf(m, 1e-10f);
        if (partials) {
            const float ys = fmaxf(yv, 1e-6f), ms = fmaxf(m, 1e-6f);
            acc += (double)(yv * logf(ys / ms) - (yv - ms));
        }
    }
    if (partials) {
        const double b = block_sum(acc);
        if (threadIdx.x == 0) partials[blockIdx.x] = b;
    }
}

__global__ void k_rl_update(float* __restrict__ x, const float* __restrict__ corr,
                            const float* __restrict__ sens, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float s = sens[i];
        const float c = s > 0.f ? corr[i] / s : 0.f;
        x[i] = fmaxf(x[i] * c, 1e-10f);
    }
}

__global__ void k_sub_floor(const float* __restrict__ y, float bg, float* __restrict__ out, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = fmaxf(y[i] - bg, 1e-6f);  // rl_mlx.py:123
}

__global__ void k_rl_mask_generic(float* __restrict__ x, float* __restrict__ sens,
                                  const double* smax, int64_t n) {
    const float fl = fmaxf((float)(*smax) * 1e-6f, 1e-10f);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float sv = sens[i];
        const bool act = sv > fl;
        sens[i] = act ? sv : 0.f;
        x[i] = act ? fmaxf(x[i], 1e-6f) : 0.f;
    }
}

__global__ void k_fill(float* __restrict__ p, float v, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        p[i] = v;
}

__global__ void k_affine(const float* __restrict__ a, float alpha, float beta,
                         float* __restrict__ out, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = alpha * a[i] + beta;
}

__global__ void k_clamp_min(const float* __restrict__ a, float lo, float* __restrict__ out, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = fmaxf(a[i], lo);
}

int hess_adjoint_tiled(const float* hw, float* out, const Dims& d, const W6& w, cudaStream_t st) {
    const int64_t grid = std::min<int64_t>(TileGeo(d).ntiles, (int64_t)sm_count() * 4);
    if (offsets_fit_u32(d))
        k_hessian_adj_t<uint32_t><<<(unsigned)std::max<int64_t>(grid, 1), 256, 0, st>>>(hw, out, d, w);
    else
        k_hessian_adj_t<int64_t><<<(unsigned)std::max<int64_t>(grid, 1), 256, 0, st>>>(hw, out, d, w);
    DK_LAUNCHED();
    return DECON_OK;
}

}  // namespace dk

using namespace dk;

// Dynamic shared-memory opt-in of a stencil kernel (once per device and
// kernel; each kernel always uses the same size) and its resident CTAs per SM.
static int smem_prepare(const void* fn, size_t bytes, int* per_sm) {
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, int> done;
    int dev = 0;
    DK_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    const auto key = std::make_pair(dev, fn);
    auto it = done.find(key);
    if (it == done.end()) {
        cudaFuncAttributes fa{};
        DK_CUDA(cudaFuncGetAttributes(&fa, fn));
        if (bytes + fa.sharedSizeBytes > 48 * 1024)  // the default covers static + dynamic
            DK_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
        DK_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     (int)cudaSharedmemCarveoutMaxShared));
        int occ = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, 256, bytes) != cudaSuccess) {
            cudaGetLastError();
            occ = 1;
        }
        it = done.emplace(key, std::max(occ, 1)).first;
    }
    if (per_sm) *per_sm = it->second;
    return DECON_OK;
}

static int g1(int64_t n) {
    return (int)std::max<int64_t>(1, std::min<int64_t>(cdiv(n, 256), (int64_t)sm_count() * 16));
}

extern "C" {

// Scalar state of a fresh solve over the history arrays at `base` (nh
// entries each, then the partial-sum slots).
static PdhgDev pdhg_initial(int num_iter, double step_scale, double delta, double eta, double tol,
                            int min_iter, int patience, double* base, int nh) {
    PdhgDev d{};
    d.tau = d.sigma = step_scale;
    d.theta = 1.0;
    d.step_scale = step_scale;
    d.delta = delta;
    d.eta = eta;
    d.tol = tol;
    d.min_iter = min_iter;
    d.patience = patience;
    d.num_iter = num_iter;
    d.final_iter = num_iter;
    d.stop = num_iter == 0 ? 1 : 0;
    d.tau_hist = base;
    d.sigma_hist = base + nh;
    d.loss_hist = base + 2 * nh;
    d.rel_hist = base + 3 * nh;
    d.partials = base + 4 * nh;
    return d;
}

int decon_pdhg_create(int num_iter, double step_scale, double delta, double eta, double tol,
                      int min_iter, int patience, decon_pdhg** out) {
    if (!out) return fail(DECON_ERR_NULL, "null pointer");
    if (num_iter < 0) return fail(DECON_ERR_VALUE, "num_iter must be >= 0");
    *out = nullptr;
    decon_pdhg* h = new (std::nothrow) decon_pdhg();
    if (!h) return fail(DECON_ERR_OOM, "host allocation failed");
    h->num_iter = num_iter;
    const int nh = std::max(num_iter, 1);
    h->capacity = nh;
    const size_t bytes = sizeof(PdhgDev) + (size_t)(4 * nh + kPdhgSlots * kPdhgGrid) * sizeof(double);
    cudaError_t e = cudaMalloc(&h->mem, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        delete h;
        return fail(DECON_ERR_OOM, "cudaMalloc of PDHG state failed: %s", cudaGetErrorString(e));
    }
    double* base = reinterpret_cast<double*>(reinterpret_cast<char*>(h->mem) + sizeof(PdhgDev));
    const PdhgDev d = pdhg_initial(num_iter, step_scale, delta, eta, tol, min_iter, patience, base, nh);
    h->dev = reinterpret_cast<PdhgDev*>(h->mem);
    // complete before the call returns: the solve may run on any stream
    int st = upload_blocking(h->dev, &d, sizeof(d));
    if (st == DECON_OK) st = memset_blocking(base, 0, (size_t)(4 * nh + kPdhgSlots * kPdhgGrid) * sizeof(double));
    if (st != DECON_OK) {
        cudaFree(h->mem);
        delete h;
        return st;
    }
    *out = h;
    return DECON_OK;
}

int decon_pdhg_reset(decon_pdhg* h, int num_iter, double step_scale, double delta, double eta,
                     double tol, int min_iter, int patience, void* stream) {
    if (!h) return fail(DECON_ERR_NULL, "null pointer");
    if (num_iter < 0) return fail(DECON_ERR_VALUE, "num_iter must be >= 0");
    const int nh = h->capacity;
    if (std::max(num_iter, 1) > nh)
        return fail(DECON_ERR_VALUE, "decon_pdhg_reset: num_iter %d exceeds the state's capacity %d",
                    num_iter, nh);
    const cudaStream_t s = as_stream(stream);
    double* base = reinterpret_cast<double*>(reinterpret_cast<char*>(h->mem) + sizeof(PdhgDev));
    const PdhgDev d = pdhg_initial(num_iter, step_scale, delta, eta, tol, min_iter, patience, base, nh);
    // pageable source: the call returns once the struct is staged
    DK_CUDA(cudaMemcpyAsync(h->dev, &d, sizeof(d), cudaMemcpyHostToDevice, s));
    DK_CUDA(cudaMemsetAsync(base, 0, (size_t)(4 * nh + kPdhgSlots * kPdhgGrid) * sizeof(double), s));
    h->num_iter = num_iter;
    return DECON_OK;
}

int decon_pdhg_destroy(decon_pdhg* h) {
    if (!h) return DECON_OK;
    cudaFree(h->mem);
    delete h;
    return DECON_OK;
}

int decon_pdhg_dual_data(decon_pdhg* h, float* y1, const float* ax_cur, const float* ax_prev,
                         const float* data, float background, int loss_type, int64_t m,
                         void* stream) {
    if (!h || !y1 || !ax_cur || !ax_prev || !data) return fail(DECON_ERR_NULL, "null pointer");
    const cudaStream_t s = as_stream(stream);
    if (loss_type == 0)
        k_dual_data<0><<<g1(m), 256, 0, s>>>(h->dev, y1, ax_cur, ax_prev, data, background, m);
    else
        k_dual_data<1><<<g1(m), 256, 0, s>>>(h->dev, y1, ax_cur, ax_prev, data, background, m);
    DK_LAUNCHED();
    return DECON_OK;
}

int decon_pdhg_dual_reg(decon_pdhg* h, float* y2, const float* lxbar, float alpha, int norm,
                        int ncomp, int64_t n, void* stream) {
    if (!h || !y2 || !lxbar) return fail(DECON_ERR_NULL, "null pointer");
    if (ncomp < 1 || ncomp > 8) return fail(DECON_ERR_VALUE, "ncomp must be 1..8");
    const cudaStream_t s = as_stream(stream);
    if (norm == 0)
        k_dual_reg<0><<<g1(n), 256, 0, s>>>(h->dev, y2, lxbar, alpha, ncomp, n);
    else
        k_dual_reg<1><<<g1(n), 256, 0, s>>>(h->dev, y2, lxbar, alpha, ncomp, n);
    DK_LAUNCHED();
    return DECON_OK;
}

int decon_pdhg_xbar(decon_pdhg* h, const float* xc, const float* xp, float* xbar, int64_t n,
                    void* stream) {
    if (!h || !xc || !xp || !xbar) return fail(DECON_ERR_NULL, "null pointer");
    k_xbar<<<g1(n), 256, 0, as_stream(stream)>>>(h->dev, xc, xp, xbar, n);
    DK_LAUNCHED();
    return DECON_OK;
}

int decon_pdhg_primal(decon_pdhg* h, const float* xc, const float* aty, const float* lty,
                      float* xn, int64_t n, void* stream) {
    if (!h || !xc || !aty || !xn) return fail(DECON_ERR_NULL, "null pointer");
    k_primal<<<kPdhgGrid, 256, 0, as_stream(stream)>>>(h->dev, xc, aty, lty, xn, n);
    DK_LAUNCHED();
    return DECON_OK;
}

int decon_pdhg_sub(decon_pdhg* h, const float* a, const float* b, float* d, int64_t n, void* stream) {
    if (!h || !a || !b || !d) return fail(DECON_ERR_NULL, "null pointer");
    k_sub<<<g1(n), 256, 0, as_stream(stream)>>>(h->dev, a, b, d, n);
    DK_LAUNCHED();
    return DECON_OK;
}

int decon_pdhg_dk(decon_pdhg* h, const float* ax_new, const float* ax_cur, int64_t m,
                  const float* l_dx, int64_t nl, void* stream) {
    if (!h || !ax_new || !ax_cur) return fail(DECON_ERR_NULL, "null pointer");
    const cudaStream_t s = as_stream(stream);
    k_diffsq_slot<<<kPdhgGrid, 256, 0, s>>>(h->dev, ax_new, ax_cur, m, kSlotDA2);
    DK_LAUNCHED();
    if (l_dx) {
        k_diffsq_slot<<<kPdhgGrid, 256, 0, s>>>(h->dev, l_dx, nullptr, nl, kSlotDL2);
        DK_LAUNCHED();
    }
    return DECON_OK;
}

int decon_pdhg_step(decon_pdhg* h, void* stream) {
    if (!h) return fail(DECON_ERR_NULL, "null pointer");
    k_step<<<1, 256, 0, as_stream(stream)>>>(h->dev);
    DK_LAUNCHED();
    return DECON_OK;
}

int decon_pdhg_loss(decon_pdhg* h, const float* ax, const float* data, float background,
                    int loss_type, int64_t m, const float* lx, int norm, int ncomp, int64_t n,
                    double alpha, int k, void* stream) {
    if (!h || !ax || !data || !lx) return fail(DECON_ERR_NULL, "null pointer");
    if (k < 0 || k >= std::max(h->num_iter, 1)) return fail(DECON_ERR_VALUE, "loss index out of range");
    const cudaStream_t s = as_stream(stream);
    if (loss_type == 0) k_loss_data<0><<<kPdhgGrid, 256, 0, s>>>(h->dev, ax, data, background, m, k);
    else k_loss_data<1><<<kPdhgGrid, 256, 0, s>>>(h->dev, ax, data, background, m, k);
    DK_LAUNCHED();
    if (norm == 0) k_loss_reg<0><<<kPdhgGrid, 256, 0, s>>>(h->dev, lx, ncomp, n, k);
    else k_loss_reg<1><<<kPdhgGrid, 256, 0, s>>>(h->dev, lx, ncomp, n, k);
    DK_LAUNCHED();
    k_record_loss<<<1, 256, 0, s>>>(h->dev, alpha, k);
    DK_LAUNCHED();
    return DECON_OK;
}

int decon_pdhg_hess_dual(decon_pdhg* h, float* y2, const float* xc, const float* xp,
                         const int64_t shape[3], float r, float alpha, int norm, void* stream) {
    if (!h || !y2 || !xc || !xp || !shape) return fail(DECON_ERR_NULL, "null pointer");
    W6 w;
    hessian_weights(r, w.w);
    const Dims d{shape[0], shape[1], shape[2]};
    const int64_t n = d.nz * d.ny * d.nx;
    (void)n;
    const TileGeo tg(d);
    int per_sm = 1;
    const void* fn = norm == 0 ? (const void*)k_hess_dual_p<0> : (const void*)k_hess_dual_p<1>;
    DK_TRY(smem_prepare(fn, DualLayout::bytes, &per_sm));
    const int grid = (int)std::min<int64_t>(tg.ntiles, (int64_t)sm_count() * per_sm);
    if (norm == 0)
        k_hess_dual_p<0><<<grid, 256, DualLayout::bytes, as_stream(stream)>>>(h->dev, y2, xc, xp, d, w, alpha);
    else
        k_hess_dual_p<1><<<grid, 256, DualLayout::bytes, as_stream(stream)>>>(h->dev, y2, xc, xp, d, w, alpha);
    DK_LAUNCHED();
    return DECON_OK;
}

int decon_pdhg_hess_primal(decon_pdhg* h, const float* xc, const float* aty, const float* y2,
                           float* xn, const int64_t shape[3], float r, void* stream) {
    if (!h || !xc || !aty || !y2 || !xn || !shape) return fail(DECON_ERR_NULL, "null pointer");
    W6 w;
    hessian_weights(r, w.w);
    const Dims d{shape[0], shape[1], shape[2]};
    if (offsets_fit_u32(d))
        k_hess_primal_t<uint32_t><<<kPdhgGrid, 256, 0, as_stream(stream)>>>(h->dev, xc, aty, y2, xn, d, w, kSlotDx2,
                                                                           kSlotXc2, kSlotXn2);
    else
        k_hess_primal_t<int64_t><<<kPdhgGrid, 256, 0, as_stream(stream)>>>(h->dev, xc, aty, y2, xn, d, w, kSlotDx2,
                                                                          kSlotXc2, kSlotXn2);
    DK_LAUNCHED();
    return DECON_OK;
}

int decon_pdhg_hess_dual_primal(decon_pdhg* h, const float* y2_in, float* y2_out, const float* xc,
                                const float* xp, const float* aty, float* xn,
                                const int64_t shape[3], float r, float alpha, int norm,
                                void* stream) {
    if (!h || !y2_in || !y2_out || !xc || !xp || !aty || !xn || !shape)
        return fail(DECON_ERR_NULL, "null pointer");
    if (y2_in == y2_out) return fail(DECON_ERR_VALUE, "y2_in and y2_out must be different buffers");
    W6 w;
    hessian_weights(r, w.w);
    const Dims d{shape[0], shape[1], shape[2]};
    const int grid = (int)std::min<int64_t>(kPdhgGrid, std::max<int64_t>(TileGeo(d).ntiles, 1));
    const cudaStream_t s = as_stream(stream);
    if (norm == 0)
        k_hess_dual_primal<0><<<grid, 256, 0, s>>>(h->dev, y2_in, y2_out, xc, xp, aty, xn, d, w, alpha,
                                                   kSlotDx2, kSlotXc2, kSlotXn2);
    else
        k_hess_dual_primal<1><<<grid, 256, 0, s>>>(h->dev, y2_in, y2_out, xc, xp, aty, xn, d, w, alpha,
                                                   kSlotDx2, kSlotXc2, kSlotXn2);
    DK_LAUNCHED();
    return DECON_OK;
}

int decon_pdhg_hess_dk(decon_pdhg* h, const float* ax_new, const float* ax_cur, int64_t m,
                       const float* xn, const float* xc, const int64_t shape[3], float r,
                       void* stream) {
    if (!h || !xn || !xc || !shape || (ax_new && !ax_cur)) return fail(DECON_ERR_NULL, "null pointer");
    W6 w;
    hessian_weights(r, w.w);
    int per_sm = 1;
    const Dims d{shape[0], shape[1], shape[2]};
    const bool u32 = offsets_fit_u32(d);
    DK_TRY(smem_prepare(u32 ? (const void*)k_hess_dk_r<uint32_t> : (const void*)k_hess_dk_r<int64_t>, 0, &per_sm));
    const int grid = (int)std::min<int64_t>(kPdhgGrid, std::max<int64_t>(TileGeo(d).ntiles, 1));
    // ax_new == NULL: only ||H dx||^2 (the data term's ||A dx||^2 then comes
    // from decon_pdhg_dk with l_dx = NULL); the empty A sum goes to the spare
    // slot 7 so that the two kernels may run concurrently
    if (u32)
        k_hess_dk_r<uint32_t><<<grid, 256, 0, as_stream(stream)>>>(h->dev, ax_new, ax_cur, ax_new ? m : 0, xn, xc,
                                                                  d, w, ax_new ? kSlotDA2 : kPdhgSlots - 1, kSlotDL2);
    else
        k_hess_dk_r<int64_t><<<grid, 256, 0, as_stream(stream)>>>(h->dev, ax_new, ax_cur, ax_new ? m : 0, xn, xc,
                                                                 d, w, ax_new ? kSlotDA2 : kPdhgSlots - 1, kSlotDL2);
    DK_LAUNCHED();
    return DECON_OK;
}

int decon_pdhg_hess_loss(decon_pdhg* h, const float* ax, const float* data, float background,
                         int loss_type, int64_t m, const float* x, const int64_t shape[3], float r,
                         int norm, double alpha, int k, void* stream) {
    if (!h || !ax || !data || !x || !shape) return fail(DECON_ERR_NULL, "null pointer");
    if (k < 0 || k >= std::max(h->num_iter, 1)) return fail(DECON_ERR_VALUE, "loss index out of range");
    W6 w;
    hessian_weights(r, w.w);
    const Dims d{shape[0], shape[1], shape[2]};
    const cudaStream_t s = as_stream(stream);
    if (loss_type == 0) k_loss_data<0><<<kPdhgGrid, 256, 0, s>>>(h->dev, ax, data, background, m, k);
    else k_loss_data<1><<<kPdhgGrid, 256, 0, s>>>(h->dev, ax, data, background, m, k);
    DK_LAUNCHED();
    int per_sm = 1;
    DK_TRY(smem_prepare(norm == 0 ? (const void*)k_hess_regloss_p<0> : (const void*)k_hess_regloss_p<1>,
                        LossLayout::bytes, &per_sm));
    const int grid = std::min(kPdhgGrid, sm_count() * per_sm);
    if (norm == 0) k_hess_regloss_p<0><<<grid, 256, LossLayout::bytes, s>>>(h->dev, x, d, w, k, kSlotReg);
    else k_hess_regloss_p<1><<<grid, 256, LossLayout::bytes, s>>>(h->dev, x, d, w, k, kSlotReg);
    DK_LAUNCHED();
    k_record_loss<<<1, 256, 0, s>>>(h->dev, alpha, k);
    DK_LAUNCHED();
    return DECON_OK;
}

int decon_pdhg_read(decon_pdhg* h, int* k, int* final_iter, int* converged, int* stop,
                    double* scalars3, double* tau_hist, double* sigma_hist, double* loss_hist,
                    double* rel_hist, void* stream) {
    if (!h) return fail(DECON_ERR_NULL, "null pointer");
    const cudaStream_t s = as_stream(stream);
    PdhgDev d;
    DK_CUDA(cudaMemcpyAsync(&d, h->dev, sizeof(d), cudaMemcpyDeviceToHost, s));
    DK_CUDA(cudaStreamSynchronize(s));
    if (k) *k = d.k;
    if (final_iter) *final_iter = d.final_iter;
    if (converged) *converged = d.converged;
    if (stop) *stop = d.stop;
    if (scalars3) {
        scalars3[0] = d.tau;
        scalars3[1] = d.sigma;
        scalars3[2] = d.theta;
    }
    const int nh = std::max(h->num_iter, 1);
    if (tau_hist) DK_CUDA(cudaMemcpy(tau_hist, d.tau_hist, nh * sizeof(double), cudaMemcpyDeviceToHost));
    if (sigma_hist) DK_CUDA(cudaMemcpy(sigma_hist, d.sigma_hist, nh * sizeof(double), cudaMemcpyDeviceToHost));
    if (loss_hist) DK_CUDA(cudaMemcpy(loss_hist, d.loss_hist, nh * sizeof(double), cudaMemcpyDeviceToHost));
    if (rel_hist) DK_CUDA(cudaMemcpy(rel_hist, d.rel_hist, nh * sizeof(double), cudaMemcpyDeviceToHost));
    return DECON_OK;
}

int decon_pdhg_status_async(decon_pdhg* h, int32_t* host_status, void* stream) {
    if (!h || !host_status) return fail(DECON_ERR_NULL, "null pointer");
    static_assert(offsetof(PdhgDev, stop) == offsetof(PdhgDev, k) + 4 * sizeof(int), "layout");
    // k, count, converged, final_iter, stop: five consecutive ints of the state
    DK_CUDA(cudaMemcpyAsync(host_status, &h->dev->k, 5 * sizeof(int), cudaMemcpyDeviceToHost,
                            as_stream(stream)));
    return DECON_OK;
}

int decon_pdhg_set_stop(decon_pdhg* h, int final_iter, void* stream) {
    if (!h) return fail(DECON_ERR_NULL, "null pointer");
    const cudaStream_t s = as_stream(stream);
    const int one = 1;
    DK_CUDA(cudaMemcpyAsync(&h->dev->stop, &one, sizeof(int), cudaMemcpyHostToDevice, s));
    DK_CUDA(cudaMemcpyAsync(&h->dev->final_iter, &final_iter, sizeof(int), cudaMemcpyHostToDevice, s));
    DK_CUDA(cudaStreamSynchronize(s));
    return DECON_OK;
}

// ---- RL for composed operators ----------------------------------------------

int decon_rl_ratio(const float* model, const float* observed, float background, float* ratio,
                   int64_t n, double* loss_sum, void* workspace, void* stream) {
    if (!model || !observed) return fail(DECON_ERR_NULL, "null pointer");
    if (loss_sum && !workspace) return fail(DECON_ERR_NULL, "loss needs a workspace");
    const cudaStream_t s = as_stream(stream);
    const int g = std::min<int>(g1(n), (int)reduce_partials_needed());
    double* part = loss_sum ? static_cast<double*>(workspace) : nullptr;
    k_rl_ratio<<<g, 256, 0, s>>>(model, observed, background, ratio, n, part);
    DK_LAUNCHED();
    if (loss_sum) DK_TRY(finish_partials(part, g, loss_sum, s));
    return DECON_OK;
}

int decon_rl_update(float* x, const float* corr, const float* sens_masked, int64_t n, void* stream) {
    if (!x || !corr || !sens_masked) return fail(DECON_ERR_NULL, "null pointer");
    k_rl_update<<<g1(n), 256, 0, as_stream(stream)>>>(x, corr, sens_masked, n);
    DK_LAUNCHED();
    return DECON_OK;
}

int decon_rl_data_floor(const float* observed, float background, float* out, int64_t n, void* stream) {
    if (!observed || !out) return fail(DECON_ERR_NULL, "null pointer");
    k_sub_floor<<<g1(n), 256, 0, as_stream(stream)>>>(observed, background, out, n);
    DK_LAUNCHED();
    return DECON_OK;
}

int decon_rl_mask(float* x, float* sens, int64_t n, void* workspace, void* stream) {
    if (!x || !sens || !workspace) return fail(DECON_ERR_NULL, "null pointer");
    const cudaStream_t s = as_stream(stream);
    double* ws = static_cast<double*>(workspace);
    // the max lands in ws[0]; partials use the rest
    DK_TRY(reduce_f32(sens, nullptr, n, DECON_RED_MAX, ws, ws + 1, reduce_partials_needed() - 1, s));
    k_rl_mask_generic<<<g1(n), 256, 0, s>>>(x, sens, ws, n);
    DK_LAUNCHED();
    return DECON_OK;
}

int decon_fill(float* p, float value, int64_t n, void* stream) {
    if (!p) return fail(DECON_ERR_NULL, "null pointer");
    if (n <= 0) return DECON_OK;
    k_fill<<<g1(n), 256, 0, as_stream(stream)>>>(p, value, n);
    DK_LAUNCHED();
    return DECON_OK;
}

int decon_affine(const float* a, float alpha, float beta, float* out, int64_t n, void* stream) {
    if (!a || !out) return fail(DECON_ERR_NULL, "null pointer");
    if (n <= 0) return DECON_OK;
    k_affine<<<g1(n), 256, 0, as_stream(stream)>>>(a, alpha, beta, out, n);
    DK_LAUNCHED();
    return DECON_OK;
}

int decon_clamp_min(const float* a, float lo, float* out, int64_t n, void* stream) {
    if (!a || !out) return fail(DECON_ERR_NULL, "null pointer");
    if (n <= 0) return DECON_OK;
    k_clamp_min<<<g1(n), 256, 0, as_stream(stream)>>>(a, lo, out, n);
    DK_LAUNCHED();
    return DECON_OK;
}

}  // extern "C"
