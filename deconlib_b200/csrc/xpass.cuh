// X passes: real-to-complex FFT of signal rows (pass 1) and complex-to-real
// FFT back to rows with the fused element-wise epilogues (pass 5).
//
// A row of Fx reals is packed as Fx/2 complex points z[n] = x[2n] + i x[2n+1]
// (even Fx), transformed with the shared-memory engine and unpacked with the
// standard split: X[k] = (Z[k] + conj Z[M-k])/2 - i W_Fx^k (Z[k] - conj Z[M-k])/2.
// Odd Fx falls back to a full complex transform of the real row.
//
// I/O: when a row is a plain, 16-byte aligned float array (Nx % 4 == 0, the
// whole signal window) each thread moves float4 vectors, several in flight,
// straight into the swizzled tile.  Points that are known zeros (the padding
// beyond Nx / 2) are never written or read: the first FFT stage of pass 1
// treats them as zeros and the last stage of pass 5 skips outputs beyond the
// crop.
#pragma once

#include "conv_impl.cuh"

namespace dk {

__device__ __forceinline__ bool kernel_src(int64_t c, int64_t F, int64_t m, int64_t npos,
                                           int64_t& k) {
    // Corner-origin embedding (utils/padding.py:142-190): canvas index c holds
    // kernel index c (c < npos) or c - F + m (the wrapped negative offsets).
    if (c < npos) {
        k = c;
        return c < m;
    }
    const int64_t nneg = m - npos;
    if (c >= F - nneg) {
        k = c - F + m;
        return true;
    }
    return false;
}

struct RowSrc {
    const float* p;  // row base (nullptr: row outside the window or constant input)
    bool ok;
};

template <int PRO>
__device__ __forceinline__ RowSrc row_source(const XR2CArgs& a, int64_t z, int64_t y) {
    RowSrc r{nullptr, false};
    if constexpr (PRO == PRO_KERNEL) {
        int64_t kz, ky;
        if (kernel_src(z, a.Nz, a.Kz, a.pz, kz) && kernel_src(y, a.Ny, a.Ky, a.py, ky)) {
            r.p = a.in + (kz * a.Ky + ky) * a.Kx;
            r.ok = true;
        }
    } else {
        const int64_t iz = z - a.win.oz, iy = y - a.win.oy;
        if (iz >= 0 && iz < a.win.wz && iy >= 0 && iy < a.win.wy) {
            r.ok = true;
            if (a.in) r.p = a.in + (iz * a.win.wy + iy) * a.win.wx;
        }
    }
    return r;
}

template <int PRO>
__device__ __forceinline__ float fetch_x(const XR2CArgs& a, const RowSrc& r, int64_t x) {
    if (!r.ok || x >= a.Nx) return 0.f;
    if constexpr (PRO == PRO_KERNEL) {
        int64_t kx;
        if (!kernel_src(x, a.Nx, a.Kx, a.px, kx)) return 0.f;
        return __ldg(r.p + kx) / a.kdiv;
    } else {
        const int64_t ix = x - a.win.ox;
        if (ix < 0 || ix >= a.win.wx) return 0.f;
        if constexpr (PRO == PRO_CONST) {
            return a.cval;
        } else if constexpr (PRO == PRO_RLINIT) {
            return fmaxf(__ldg(r.p + ix) - a.bg, 1e-6f);
        } else {
            return __ldg(r.p + ix);
        }
    }
}

// ---------------------------------------------------------------------------
// pass 1: X R2C
// ---------------------------------------------------------------------------

// Lines per CTA of the X passes for a compile-time length (the host's rule,
// fft_lines_per_cta: T x L <= kSmemElems complex values and T x ceil(L / 32)
// <= kFftThreads threads, T <= 32, a power of two).
__host__ __device__ constexpr int x_lines(int LS) {
    int T = 1;
    while (T * 2 <= 32 && T * 2 * LS <= kSmemElems && T * 2 * ((LS + 31) / 32) <= kFftThreads) T *= 2;
    return T;
}

template <int PRO, int LS>
__global__ void __launch_bounds__(LS > 0 ? kFftThreads : kDynThreads, LS > 0 ? 3 : 1) k_xr2c(XR2CArgs a) {
    extern __shared__ float2 sm[];
    __shared__ RowSrc rsrc[32];  // per-row source (general path)
    constexpr int TC = LS > 0 ? x_lines(LS) : 0;  // compile-time lines per CTA
    const int T = TC > 0 ? TC : a.T, L = LS > 0 ? LS : a.ax.L, tid = threadIdx.x;
    auto phys = [&](int j, int t, int) { return physw<TC>(j, t, T); };
    const int64_t row0 = (int64_t)blockIdx.x * T;
    // packed points that can be non-zero
    const int nin = a.odd ? (int)(a.Nx < L ? a.Nx : L) : (int)(((a.Nx + 1) >> 1) < L ? ((a.Nx + 1) >> 1) : L);
    if constexpr (PRO == PRO_UP2) {
        // fine row (z, y) of the adjoint of the 2x area sum: fine x = 2n and
        // 2n + 1 both take coarse value n of coarse row (z / 2, y / 2), so the
        // packed point n is (c[n], c[n]) (even Fx, even extents)
        const int64_t mx = a.Nx >> 1, my = a.Ny >> 1;
        if (a.vec4) {
            // four coarse values (one float4) per thread step, several in flight
            const int q4 = (int)(mx >> 2), nq = T * q4;
            constexpr int U = 4;
            #pragma unroll 1
            for (int c0 = tid; c0 < nq; c0 += U * blockDim.x) {
                float4 v[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int c = c0 + u * blockDim.x;
                    const int t = fdiv(c, a.fd_q4);
                    const int64_t row = row0 + t;
                    float4 w = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (c < nq && row < a.nrows) {
                        const int64_t z = row / a.Ny, y = row - z * a.Ny;
                        w = __ldg(reinterpret_cast<const float4*>(a.in + ((z >> 1) * my + (y >> 1)) * mx) +
                                  (c - t * q4));
                    }
                    v[u] = w;
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int c = c0 + u * blockDim.x;
                    if (c < nq) {
                        const int t = fdiv(c, a.fd_q4), n = 4 * (c - t * q4);
                        sm[phys(n, t, T)] = make_float2(v[u].x, v[u].x);
                        sm[phys(n + 1, t, T)] = make_float2(v[u].y, v[u].y);
                        sm[phys(n + 2, t, T)] = make_float2(v[u].z, v[u].z);
                        sm[phys(n + 3, t, T)] = make_float2(v[u].w, v[u].w);
                    }
                }
            }
        } else {
        #pragma unroll 1
        for (int q = tid; q < T * nin; q += blockDim.x) {
            const int t = fdiv(q, a.fd_nin), n = q - t * nin;
            const int64_t row = row0 + t;
            float v = 0.f;
            if (row < a.nrows) {
                const int64_t z = row / a.Ny, y = row - z * a.Ny;
                v = __ldg(a.in + ((z >> 1) * my + (y >> 1)) * mx + n);
            }
            sm[phys(n, t, T)] = make_float2(v, v);
        }
        }
    } else if (PRO == PRO_ARRAY && a.vec4) {
        const int q4 = (int)(a.Nx >> 2);  // float4 per row
        const int nq = T * q4;
        constexpr int U = 4;
        #pragma unroll 1
        for (int c0 = tid; c0 < nq; c0 += U * blockDim.x) {
            float4 v[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int c = c0 + u * blockDim.x;
                const int t = fdiv(c, a.fd_q4);
                const int64_t row = row0 + t;
                v[u] = (c < nq && row < a.nrows)
                           ? __ldg(reinterpret_cast<const float4*>(a.in + row * a.Nx) + (c - t * q4))
                           : make_float4(0.f, 0.f, 0.f, 0.f);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int c = c0 + u * blockDim.x;
                if (c < nq) {
                    const int t = fdiv(c, a.fd_q4), x4 = c - t * q4;
                    sm[phys(2 * x4, t, T)] = make_float2(v[u].x, v[u].y);
                    sm[phys(2 * x4 + 1, t, T)] = make_float2(v[u].z, v[u].w);
                }
            }
        }
    } else {
        // (z, y) of each row once, not per element
        if (tid < T) {
            const int64_t row = row0 + tid;
            RowSrc rs{nullptr, false};
            if (row < a.nrows) {
                const int64_t z = row / a.Ny, y = row - z * a.Ny;
                rs = row_source<PRO>(a, z, y);
            }
            rsrc[tid] = rs;
        }
        __syncthreads();
        #pragma unroll 1
        for (int q = tid; q < T * nin; q += blockDim.x) {
            const int t = fdiv(q, a.fd_nin), n = q - t * nin;
            const RowSrc rs = rsrc[t];
            float2 v = make_float2(0.f, 0.f);
            if (a.odd) {
                v.x = fetch_x<PRO>(a, rs, n);
            } else {
                v.x = fetch_x<PRO>(a, rs, 2 * (int64_t)n);
                v.y = fetch_x<PRO>(a, rs, 2 * (int64_t)n + 1);
            }
            sm[phys(n, t, T)] = v;
        }
    }
    if constexpr (LS == 0) {
        // the runtime-radix path reads every point: zero the padding
        const int nz = L - nin;
        #pragma unroll 1
        for (int q = tid; q < T * nz; q += blockDim.x) {
            const int t = q / nz;
            sm[phys(nin + (q - t * nz), t, T)] = make_float2(0.f, 0.f);
        }
    }
    __syncthreads();
    if constexpr (LS > 0) fft_lines_static<LS, -1, 1, TC>(sm, T, tid % T, tid / T, a.ax.tw, a.ax.tws, nin);
    else fft_lines<-1, LS>(sm, T, tid % T, tid / T, a.ax, nin);
    const int H = a.Hx;
    const int lgT = 31 - __clz(T);  // T is a power of two
    if (a.odd) {
        #pragma unroll 1
        for (int q = tid; q < T * H; q += blockDim.x) {
            int t, k;
            if (a.kstride) {
                k = q >> lgT;
                t = q & (T - 1);
            } else {
                t = fdiv(q, a.fd_H);
                k = q - t * H;
            }
            const int64_t row = row0 + t;
            if (row < a.nrows) a.out[a.kstride ? k * a.kstride + row : row * a.P + k] = sm[phys(k, t, T)];
        }
    } else if (a.kstride) {
        // kx-major spectrum: consecutive threads take consecutive rows at one
        // frequency pair, so every warp stores two 256-byte runs
        const int M = L, np = (M >> 1) + 1;
        #pragma unroll 1
        for (int q = tid; q < T * np; q += blockDim.x) {
            const int k = q >> lgT, t = q & (T - 1);
            const int64_t row = row0 + t;
            if (row >= a.nrows) continue;
            const int km = M - k;
            const float2 zk = sm[phys(k, t, T)];
            const float2 zm = cconj(sm[phys(k == 0 ? 0 : km, t, T)]);
            const float2 e = cscale(cadd(zk, zm), 0.5f);
            const float2 o = rot90<-1>(cscale(csub(zk, zm), 0.5f));
            if (k < H) a.out[k * a.kstride + row] = cadd(e, cmul(__ldg(&a.twx[k]), o));
            if (km != k && km < H) a.out[km * a.kstride + row] = cadd(cconj(e), cmul(__ldg(&a.twx[km]), cconj(o)));
        }
    } else {
        // X[k] = e + W^k o and X[M-k] = conj(e) + W^(M-k) conj(o) with
        // e = (Z[k] + conj Z[M-k]) / 2, o = -i (Z[k] - conj Z[M-k]) / 2: one
        // thread per pair (k, M - k), the same float operations as the
        // single-output form (X[M] pairs with X[0], indices mod M).
        const int M = L, np = (M >> 1) + 1;
        #pragma unroll 1
        for (int q = tid; q < T * np; q += blockDim.x) {
            const int t = fdiv(q, a.fd_np), k = q - t * np;
            const int64_t row = row0 + t;
            if (row >= a.nrows) continue;
            const int km = M - k;  // partner output (M for k = 0)
            const float2 zk = sm[phys(k, t, T)];
            const float2 zm = cconj(sm[phys(k == 0 ? 0 : km, t, T)]);
            const float2 e = cscale(cadd(zk, zm), 0.5f);
            const float2 o = rot90<-1>(cscale(csub(zk, zm), 0.5f));
            float2* orow = a.out + row * a.P;
            if (k < H) orow[k] = cadd(e, cmul(__ldg(&a.twx[k]), o));
            if (km != k && km < H) orow[km] = cadd(cconj(e), cmul(__ldg(&a.twx[km]), cconj(o)));
        }
    }
}

// ---------------------------------------------------------------------------
// pass 5: X C2R with fused epilogues
// ---------------------------------------------------------------------------

// Spectrum row of the CTA's line t: rows blockIdx.x * T + t, or, for the 2x
// area-sum epilogue, lines t < T / 2 from plane 2k and lines t >= T / 2 from
// plane 2k + 1 over the same T / 2 y values, so that each CTA holds whole
// 2 x 2 x 2 blocks.
template <int EPI>
__device__ __forceinline__ int64_t c2r_row(const XC2RArgs& a, int T, int t) {
    if constexpr (EPI == EPI_DOWN2) {
        const int h = T >> 1;
        const int64_t b = blockIdx.x, nyb = a.Ny / h;
        const int64_t k = b / nyb, yb = b - k * nyb;
        return (2 * k + (t >= h ? 1 : 0)) * a.Ny + yb * h + (t & (h - 1));
    } else {
        return (int64_t)blockIdx.x * T + t;
    }
}

// The element-wise epilogue on one output voxel i (v already scaled).
template <int EPI>
__device__ __forceinline__ void epilogue(const XC2RArgs& a, int64_t i, float v, double& acc) {
    if constexpr (EPI == EPI_STORE) {
        a.out[i] = v;
    } else if constexpr (EPI == EPI_RL_RATIO || EPI == EPI_PRED) {
        // rl_mlx.py:147-148  model = A x + b ; ratio = y / max(model, 1e-10)
        const float m = v + a.bg;
        const float yv = __ldg(a.aux0 + i);
        if constexpr (EPI == EPI_RL_RATIO) {
            a.out[i] = yv / fmaxf(m, 1e-10f);
        } else {
            a.out[i] = m;
        }
        if (a.partials) {
            // rl_mlx.py:75-79: y log(max(y,eps)/max(m,eps)) - (y - max(m,eps))
            const float ys = fmaxf(yv, 1e-6f), ms = fmaxf(m, 1e-6f);
            acc += (double)(yv * logf(ys / ms) - (yv - ms));
        }
    } else if constexpr (EPI == EPI_RL_UPDATE) {
        // rl_mlx.py:149-150  x = max(x * where(active, A^T ratio / sens, 0), 1e-10)
        const float s = __ldg(a.aux1 + i);
        const float c = s > 0.f ? v / s : 0.f;
        a.out[i] = fmaxf(a.aux0[i] * c, 1e-10f);
    }
}

// Three CTAs per SM below length 512 (80 registers, no spills; at 256 the
// PDHG iteration measured 1.04-1.05 vs 1.06-1.07 ms with two); from 512 on
// the compile-time lines per CTA need more registers, so two.
template <int EPI, int LS>
__global__ void __launch_bounds__(LS > 0 ? kFftThreads : kDynThreads, LS > 0 ? (LS < 512 ? 3 : 2) : 1) k_xc2r(XC2RArgs a) {
    extern __shared__ float2 sm[];
    __shared__ float2 nyq[32];    // X[M] of each row (even Fx)
    __shared__ int64_t obase[32];  // output index of x = 0 of each row (general path)
    constexpr int64_t kOutside = INT64_MIN;
    // compile-time lines per CTA from L = 512 on (measured 211 -> 198 us at
    // Fx = 1024); at L = 256 it brought no gain and spilled the loss epilogues
    constexpr int TC = LS >= 512 ? x_lines(LS) : 0;
    const int T = TC > 0 ? TC : a.T, L = LS > 0 ? LS : a.ax.L, tid = threadIdx.x;
    auto phys = [&](int j, int t, int) { return physw<TC>(j, t, T); };
    const int64_t row0 = (int64_t)blockIdx.x * T;
    const int lgT = 31 - __clz(T);  // T is a power of two
    if (a.odd) {
        #pragma unroll 1
        for (int q = tid; q < T * L; q += blockDim.x) {
            int t, k;
            if (a.kstride) {
                k = q >> lgT;
                t = q & (T - 1);
            } else {
                t = fdiv(q, a.fd_L);
                k = q - t * L;
            }
            const int64_t row = c2r_row<EPI>(a, T, t);
            float2 Z = make_float2(0.f, 0.f);
            if (row < a.nrows) {
                // full Hermitian spectrum from the half: X[k] = conj(X[Fx - k])
                if (a.kstride) {
                    Z = k < a.Hx ? a.in[k * a.kstride + row] : cconj(a.in[(L - k) * a.kstride + row]);
                } else {
                    const float2* rp = a.in + row * a.P;
                    Z = k < a.Hx ? rp[k] : cconj(rp[L - k]);
                }
                if (k == 0) Z.y = 0.f;
            }
            sm[phys(k, t, T)] = Z;
        }
        __syncthreads();
    } else {
        const int M = L;
        if (a.kstride) {
            // kx-major spectrum: a warp reads 32 consecutive rows of one
            // frequency (256 bytes) per load
            #pragma unroll 1
            for (int q = tid; q < T * M; q += blockDim.x) {
                const int k = q >> lgT, t = q & (T - 1);
                const int64_t row = c2r_row<EPI>(a, T, t);
                sm[phys(k, t, T)] = row < a.nrows ? a.in[k * a.kstride + row] : make_float2(0.f, 0.f);
            }
            #pragma unroll 1
            for (int t = tid; t < T; t += blockDim.x) {
                const int64_t row = c2r_row<EPI>(a, T, t);
                nyq[t] = row < a.nrows ? a.in[M * a.kstride + row] : make_float2(0.f, 0.f);
            }
        } else {
            // stage the half spectrum: X[0..M) as float4 pairs, X[M] aside
            const int h2 = M >> 1;  // float4 (two complex) per row
            const int nq = T * h2;
            constexpr int U = 4;
            #pragma unroll 1
            for (int c0 = tid; c0 < nq; c0 += U * blockDim.x) {
                float4 v[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int c = c0 + u * blockDim.x;
                    const int t = fdiv(c, a.fd_h2);
                    const int64_t row = c2r_row<EPI>(a, T, t);
                    v[u] = (c < nq && row < a.nrows)
                               ? __ldg(reinterpret_cast<const float4*>(a.in + row * a.P) + (c - t * h2))
                               : make_float4(0.f, 0.f, 0.f, 0.f);
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int c = c0 + u * blockDim.x;
                    if (c < nq) {
                        const int t = fdiv(c, a.fd_h2), q2 = c - t * h2;
                        sm[phys(2 * q2, t, T)] = make_float2(v[u].x, v[u].y);
                        sm[phys(2 * q2 + 1, t, T)] = make_float2(v[u].z, v[u].w);
                    }
                }
            }
            #pragma unroll 1
            for (int t = tid; t < T; t += blockDim.x) {
                const int64_t row = c2r_row<EPI>(a, T, t);
                const bool ok = row < a.nrows;
                nyq[t] = ok ? a.in[row * a.P + M] : make_float2(0.f, 0.f);
                // odd M: the last packed point is not covered by the float4 pairs
                if (M & 1) sm[phys(M - 1, t, T)] = ok ? a.in[row * a.P + M - 1] : make_float2(0.f, 0.f);
            }
        }
        __syncthreads();
        // Z[k] = (X[k] + conj X[M-k]) + i (X[k] - conj X[M-k]) W_Fx^-k, one
        // thread per pair (k, M - k); irfft ignores Im of DC and Nyquist.
        const int npair = (M >> 1) + 1;
        #pragma unroll 1
        for (int q = tid; q < T * npair; q += blockDim.x) {
            const int t = fdiv(q, a.fd_npair), k = q - t * npair;
            if (k == 0) {
                float2 x0 = sm[phys(0, t, T)], xm = nyq[t];
                x0.y = 0.f;
                xm.y = 0.f;
                xm = cconj(xm);
                const float2 e = cadd(x0, xm);
                const float2 od = cmulc(csub(x0, xm), __ldg(&a.twx[0]));
                sm[phys(0, t, T)] = cadd(e, rot90<+1>(od));
            } else {
                const int km = M - k;
                const float2 xk = sm[phys(k, t, T)];
                const float2 xm = sm[phys(km, t, T)];
                {
                    const float2 c2 = cconj(xm);
                    const float2 e = cadd(xk, c2);
                    const float2 od = cmulc(csub(xk, c2), __ldg(&a.twx[k]));
                    sm[phys(k, t, T)] = cadd(e, rot90<+1>(od));
                }
                if (km != k) {
                    const float2 c2 = cconj(xk);
                    const float2 e = cadd(xm, c2);
                    const float2 od = cmulc(csub(xm, c2), __ldg(&a.twx[km]));
                    sm[phys(km, t, T)] = cadd(e, rot90<+1>(od));
                }
            }
        }
        __syncthreads();
    }
    // outputs beyond the kept x range are not needed
    const int nout = a.odd ? (int)(a.Nx < L ? a.Nx : L) : (int)(((a.Nx + 1) >> 1) < L ? ((a.Nx + 1) >> 1) : L);
    if constexpr (LS > 0) fft_lines_static<LS, +1, 1, TC>(sm, T, tid % T, tid / T, a.ax.tw, a.ax.tws, 1 << 30, nout);
    else fft_lines<+1, LS>(sm, T, tid % T, tid / T, a.ax, 1 << 30, nout);

    double acc = 0.0;
    const int64_t Nx = a.Nx;
    if constexpr (EPI == EPI_DOWN2) {
        // 2x area sum of the scaled output, in the order of the three banded
        // passes (z pairs, then y pairs, then x pairs; unit weights): line t
        // holds plane 2k (t < T/2) or 2k + 1, packed point i holds x = 2i, 2i + 1
        const int h = T >> 1, hq = h >> 1;
        const int64_t mx = Nx >> 1, my = a.Ny >> 1;
        const int64_t nyb = a.Ny / h, k = (int64_t)blockIdx.x / nyb, yb = (int64_t)blockIdx.x - k * nyb;
        const int nq = hq * (int)mx;
        const float s = a.scale;
        #pragma unroll 1
        for (int q = tid; q < nq; q += blockDim.x) {
            const int j = fdiv(q, a.fd_q4), i = q - j * (int)mx;  // fd_q4 holds mx here
            const float2 p0 = sm[phys(i, 2 * j, T)], p1 = sm[phys(i, 2 * j + 1, T)];
            const float2 q0 = sm[phys(i, h + 2 * j, T)], q1 = sm[phys(i, h + 2 * j + 1, T)];
            // round-to-nearest intrinsics: every product and sum rounded as
            // the stored output and the separate passes round it (no fma)
            const float a0x = __fadd_rn(__fmul_rn(p0.x, s), __fmul_rn(q0.x, s));  // z pairs, y = 2j
            const float a0y = __fadd_rn(__fmul_rn(p0.y, s), __fmul_rn(q0.y, s));
            const float a1x = __fadd_rn(__fmul_rn(p1.x, s), __fmul_rn(q1.x, s));  // y = 2j + 1
            const float a1y = __fadd_rn(__fmul_rn(p1.y, s), __fmul_rn(q1.y, s));
            const float bx = __fadd_rn(a0x, a1x), by = __fadd_rn(a0y, a1y);       // y pairs
            a.out[(k * my + yb * hq + j) * mx + i] = __fadd_rn(bx, by);           // x pair
        }
    } else if (a.vec4) {
        // plain rows, full window: 4 voxels per thread step
        const int q4 = (int)(Nx >> 2), nq = T * q4;
        #pragma unroll 1
        for (int c = tid; c < nq; c += blockDim.x) {
            const int t = fdiv(c, a.fd_q4), x4 = c - t * q4;
            const int64_t row = c2r_row<EPI>(a, T, t);
            if (row >= a.nrows) continue;
            const float2 p0 = sm[phys(2 * x4, t, T)], p1 = sm[phys(2 * x4 + 1, t, T)];
            const int64_t i = row * Nx + 4 * x4;
            const float s = a.scale;
            if constexpr (EPI == EPI_STORE) {
                *reinterpret_cast<float4*>(a.out + i) = make_float4(p0.x * s, p0.y * s, p1.x * s, p1.y * s);
            } else if constexpr (EPI == EPI_RL_UPDATE) {
                const float4 sv = __ldg(reinterpret_cast<const float4*>(a.aux1 + i));
                const float4 xv = *reinterpret_cast<const float4*>(a.aux0 + i);
                const float v[4] = {p0.x * s, p0.y * s, p1.x * s, p1.y * s};
                const float ss[4] = {sv.x, sv.y, sv.z, sv.w};
                const float xx[4] = {xv.x, xv.y, xv.z, xv.w};
                float o[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const float cc = ss[e] > 0.f ? v[e] / ss[e] : 0.f;
                    o[e] = fmaxf(xx[e] * cc, 1e-10f);
                }
                *reinterpret_cast<float4*>(a.out + i) = make_float4(o[0], o[1], o[2], o[3]);
            } else {
                const float4 yv = __ldg(reinterpret_cast<const float4*>(a.aux0 + i));
                const float v[4] = {p0.x * s, p0.y * s, p1.x * s, p1.y * s};
                const float yy[4] = {yv.x, yv.y, yv.z, yv.w};
                float o[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const float m = v[e] + a.bg;
                    o[e] = EPI == EPI_RL_RATIO ? yy[e] / fmaxf(m, 1e-10f) : m;
                    if (a.partials) {
                        const float ys = fmaxf(yy[e], 1e-6f), ms = fmaxf(m, 1e-6f);
                        acc += (double)(yy[e] * logf(ys / ms) - (yy[e] - ms));
                    }
                }
                *reinterpret_cast<float4*>(a.out + i) = make_float4(o[0], o[1], o[2], o[3]);
            }
        }
    } else {
        // window rows: output index of x = 0 per row, once
        if (tid < T) {
            const int64_t row = c2r_row<EPI>(a, T, tid);
            int64_t b = kOutside;
            if (row < a.nrows) {
                const int64_t z = row / a.Ny, y = row - z * a.Ny;
                const int64_t iz = z - a.win.oz, iy = y - a.win.oy;
                if (iz >= 0 && iz < a.win.wz && iy >= 0 && iy < a.win.wy)
                    b = (iz * a.win.wy + iy) * a.win.wx - a.win.ox;
            }
            obase[tid] = b;
        }
        __syncthreads();
        const int nx = (int)Nx;
        #pragma unroll 1
        for (int q = tid; q < T * nx; q += blockDim.x) {
            const int t = fdiv(q, a.fd_Nx);
            const int x = q - t * nx;
            const int64_t b = obase[t];
            const int64_t ix = x - a.win.ox;
            if (b == kOutside || ix < 0 || ix >= a.win.wx) continue;
            float v;
            if (a.odd) {
                v = sm[phys(x, t, T)].x;
            } else {
                const float2 c = sm[phys(x >> 1, t, T)];
                v = (x & 1) ? c.y : c.x;
            }
            epilogue<EPI>(a, b + x, v * a.scale, acc);
        }
    }
    if constexpr (EPI == EPI_RL_RATIO || EPI == EPI_PRED) {
        if (a.partials) {
            const double s = block_sum(acc);
            if (tid == 0) a.partials[blockIdx.x] = s;
        }
    }
}

}  // namespace dk
