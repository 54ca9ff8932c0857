// Persistent, software-pipelined column FFT pass (Y and axial passes).
//
// Each CTA loops over 16-column tiles (tile i, i + grid, ...).  Tiles arrive
// through an NS-deep ring of TMA loads (one mbarrier per ring slot, bounded
// waits), so the next tiles stream in while the current one is transformed.
// The transform of a line of L = SPLIT * R * R points runs as two radix-R
// Stockham stages with K = 1 butterfly per thread per stage: thread (t, j)
// owns column t and butterfly j in both stages, so the second-stage twiddles
// W_{R^2}^{r j} are computed once per thread and stay in registers.
//
// SPLIT = 2 uses the half-zero structure of the canvas (the signal occupies at
// most half of the axis):
//   forward, x[n] = 0 for n >= L/2:  X[2m] = FFT_{L/2}(x)[m],
//                                     X[2m+1] = FFT_{L/2}(x[n] W_L^n)[m];
//   inverse, only y[n], n < L/2, kept: y[n] = IFFT_{L/2}(X[2m])[n]
//                                     + W_L^{-n} IFFT_{L/2}(X[2m+1])[n].
// The axial pass (MODE = COL_OTF / COL_OTF_CONJ) multiplies by the OTF in
// registers between the forward and inverse transforms: after the forward
// second stage a thread holds X at m = j + R r, exactly the points the inverse
// first stage needs.  The FP32 OTF tile (L rows x 16 columns) arrives by TMA
// in the same ring slot and on the same mbarrier as the spectrum tile, so its
// loads run NS tiles ahead like the spectrum's; the FP16 OTF of the
// mixed-precision mode is prefetched from global memory into registers
// before the tile's barrier wait.
#pragma once

#include "conv_impl.cuh"
#include "tma.cuh"

namespace dk {

__device__ __forceinline__ int p1(int row, int t) { return physw<1>(row, t, 16); }

// Ring slots of k_col_pipe (the host sizes shared memory with the same rule).
__host__ __device__ constexpr int pipe_slots(int L, bool lean) { return lean ? 2 : (L >= 512 ? 2 : 3); }

// H16: the OTF is read from the FP16 copy and rescaled per kz plane (mixed
// precision); the transforms and the product stay FP32.
// LEAN: twiddles in shared memory instead of registers, one ring slot,
// <= 128 registers, so two CTAs share an SM and one CTA's barriers and loads
// overlap the other's arithmetic.
template <int R, int SPLIT, int MODE, bool H16 = false, bool LEAN = false>
__global__ void __launch_bounds__(16 * R, LEAN ? 2 : 1) k_col_pipe(const __grid_constant__ PipeArgs a) {
    constexpr int LH = R * R;          // sub-transform length
    constexpr int L = LH * SPLIT;      // axis length
    constexpr int NS = pipe_slots(L, LEAN);
    constexpr bool OTF = (MODE == COL_OTF || MODE == COL_OTF_CONJ);
    constexpr bool INV_FIRST = (MODE == COL_INV);
    constexpr bool OTFT = OTF && !H16;              // FP32 OTF tile staged by TMA
    // LEAN axial pass: one OTF buffer (FP32, or FP16 under H16) beside a
    // two-slot spectrum ring, loaded for the next tile as soon as the current
    // tile's product is done
    constexpr bool OTF1 = OTF && LEAN;
    constexpr bool OTF1H = OTF1 && H16;             // FP16 OTF tile staged by TMA
    constexpr int SLOT = L * 16 * (OTFT && !OTF1 ? 2 : 1);  // float2 per ring slot
    constexpr int D1 = INV_FIRST ? +1 : -1;  // direction of the first transform
    extern __shared__ unsigned char smraw[];
    float2* base = reinterpret_cast<float2*>((reinterpret_cast<uintptr_t>(smraw) + 1023) & ~uintptr_t(1023));
    __shared__ uint64_t full[NS];
    __shared__ uint64_t obar;  // OTF1: the OTF buffer arrived
    const int tid = threadIdx.x, t = tid & 15, j = tid >> 4;
    const int total = a.nouter * a.ntiles;

    // second-stage twiddles W_LH^(r j) = W_L^(SPLIT r j): registers, or (LEAN)
    // a shared [R][R] table filled before the first barrier
    float2 w2r[LEAN ? 1 : R];
    __shared__ float2 w2s[LEAN ? R : 1][LEAN ? R : 1];
    if constexpr (LEAN) {
        for (int q = tid; q < R * R; q += blockDim.x) w2s[q / R][q % R] = __ldg(&a.tw[(SPLIT * (q / R) * (q % R)) * a.tws]);
    } else {
#pragma unroll
        for (int r = 0; r < R; ++r) w2r[r] = __ldg(&a.tw[(SPLIT * r * j) * a.tws]);
    }
    auto w2 = [&](int r) -> float2 {
        if constexpr (LEAN) return w2s[r][j];
        else return w2r[r];
    };
    // split twiddles W_L^n, n = j + R r: registers, or (LEAN) a shared table
    float2 wsr[SPLIT == 2 && !LEAN ? R : 1];
    __shared__ float2 wss[SPLIT == 2 && LEAN ? R * R : 1];
    if constexpr (SPLIT == 2) {
        if constexpr (LEAN) {
            for (int q = tid; q < R * R; q += blockDim.x) wss[q] = __ldg(&a.tw[q * a.tws]);
        } else {
#pragma unroll
            for (int r = 0; r < R; ++r) wsr[r] = __ldg(&a.tw[(j + R * r) * a.tws]);
        }
    }
    auto ws = [&](int r) -> float2 {
        if constexpr (LEAN) return wss[j + R * r];
        else return wsr[SPLIT == 2 ? r : 0];
    };

    // FP16 OTF: this thread's kz planes are fixed, so are their scales
    float os[H16 && !LEAN ? SPLIT : 1][H16 && !LEAN ? R : 1];
    __shared__ float oss[OTF1H ? L : 1];  // OTF1H: the scales of all L kz planes
    if constexpr (OTF1H) {
        for (int q = tid; q < L; q += blockDim.x) oss[q] = __ldg(a.otf_inv + q);
    } else if constexpr (H16) {
#pragma unroll
        for (int h = 0; h < SPLIT; ++h)
#pragma unroll
            for (int r = 0; r < R; ++r) os[h][r] = __ldg(a.otf_inv + SPLIT * (j + R * r) + h);
    }

    float2* otf1 = base + NS * SLOT;  // OTF1 buffer
    const __half2* otf1h = reinterpret_cast<const __half2*>(otf1);  // OTF1H view: [L][16] half2
    if (tid == 0) {
        for (int s = 0; s < NS; ++s) mbar_init(&full[s], 1);
        if constexpr (OTF1) mbar_init(&obar, 1);
        fence_proxy_async_smem();
    }
    __syncthreads();
    const int nbox = (a.nin + a.src_box - 1) / a.src_box;
    auto issue = [&](int tile, int s) {
        const int o = tile / a.ntiles;
        const int c0 = (tile - o * a.ntiles) * 32;
        float2* buf = base + s * SLOT;
        mbar_expect_tx(&full[s], (uint32_t)(nbox * a.src_box * 128) + (OTFT && !OTF1 ? (uint32_t)(L * 128) : 0u));
        for (int i = 0; i < nbox; ++i) {
            const int r0 = i * a.src_box;
            if (a.src_jdim == 1) tma_load_3d(buf + r0 * 16, &a.src, c0, r0, o, &full[s]);
            else tma_load_3d(buf + r0 * 16, &a.src, c0, o, r0, &full[s]);
        }
        if constexpr (OTFT && !OTF1)
            for (int r0 = 0; r0 < L; r0 += a.otf_box) tma_load_3d(buf + L * 16 + r0 * 16, &a.otfmap, c0, o, r0, &full[s]);
    };
    auto issue_otf = [&](int tile) {
        const int o = tile / a.ntiles;
        const int c0 = (tile - o * a.ntiles) * 32;
        if constexpr (OTF1H) {
            // half2 elements: column c0 / 2, rows of 64 bytes
            mbar_expect_tx(&obar, (uint32_t)(L * 64));
            for (int r0 = 0; r0 < L; r0 += a.otf_box)
                tma_load_3d(reinterpret_cast<__half2*>(otf1) + r0 * 16, &a.otfmap16, c0 >> 1, o, r0, &obar);
        } else {
            mbar_expect_tx(&obar, (uint32_t)(L * 128));
            for (int r0 = 0; r0 < L; r0 += a.otf_box) tma_load_3d(otf1 + r0 * 16, &a.otfmap, c0, o, r0, &obar);
        }
    };
    if (tid == 0) {
        for (int s = 0; s < NS; ++s) {
            const int tile = blockIdx.x + s * gridDim.x;
            if (tile < total) issue(tile, s);
        }
        if constexpr (OTF1)
            if ((int)blockIdx.x < total) issue_otf(blockIdx.x);
    }

    for (int it = 0;; ++it) {
        const int tile = blockIdx.x + it * gridDim.x;
        if (tile >= total) break;
        const int s = it % NS;
        const uint32_t ph = (uint32_t)((it / NS) & 1);
        float2* buf = base + s * SLOT;
        const float2* obuf = OTF1 ? otf1 : buf + L * 16;  // OTF tile (OTFT)
        const int o = tile / a.ntiles;
        const int c0 = (tile - o * a.ntiles) * 32;

        (void)obuf;
        // FP16 OTF (H16): raw values and plane scales are only loaded here and
        // converted where they are used, so the loads stay in flight across
        // the tile wait and the forward transform like the FP32 ones.
        __half2 oh[H16 && !LEAN ? SPLIT : 1][H16 && !LEAN ? R : 1];
        if constexpr (OTF && H16 && !LEAN) {
            const __half2* op = a.otf16 + o * a.otf_os + (c0 >> 1) + t;
#pragma unroll
            for (int h = 0; h < SPLIT; ++h)
#pragma unroll
                for (int r = 0; r < R; ++r) oh[h][r] = __ldg(op + (int64_t)(SPLIT * (j + R * r) + h) * a.otf_js);
        }
        if (!__syncthreads_and(mbar_wait_bounded(&full[s], ph))) return;

        float2 v[SPLIT][R];
        // ---- stage 1 of the first transform (Ns = 1) ----
        if constexpr (!INV_FIRST) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int n = j + R * r;
                const float2 x = n < a.nin ? buf[p1(n, t)] : make_float2(0.f, 0.f);
                v[0][r] = x;
                if constexpr (SPLIT == 2) v[1][r] = cmul(x, ws(r));
            }
        } else {
#pragma unroll
            for (int h = 0; h < SPLIT; ++h)
#pragma unroll
                for (int r = 0; r < R; ++r) v[h][r] = buf[p1(SPLIT * (j + R * r) + h, t)];
        }
#pragma unroll
        for (int h = 0; h < SPLIT; ++h) dft<R, D1>(v[h]);
        __syncthreads();
#pragma unroll
        for (int h = 0; h < SPLIT; ++h)
#pragma unroll
            for (int r = 0; r < R; ++r) buf[p1(h * LH + j * R + r, t)] = v[h][r];
        __syncthreads();
        // ---- stage 2 (Ns = R): reads and writes point j + R r ----
#pragma unroll
        for (int h = 0; h < SPLIT; ++h) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const float2 x = buf[p1(h * LH + j + R * r, t)];
                v[h][r] = r == 0 ? x : (D1 < 0 ? cmul(x, w2(r)) : cmulc(x, w2(r)));
            }
            dft<R, D1>(v[h]);
        }
        if constexpr (OTF) {
            if constexpr (OTF1)
                if (!__syncthreads_and(mbar_wait_bounded(&obar, (uint32_t)(it & 1)))) return;
            // X at m = j + R r  ->  x OTF  ->  inverse stage 1 in registers
#pragma unroll
            for (int h = 0; h < SPLIT; ++h) {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    float2 w;
                    if constexpr (OTF1H) {
                        const int kz = SPLIT * (j + R * r) + h;
                        const float2 q = __half22float2(otf1h[kz * 16 + t]);
                        w = make_float2(q.x * oss[kz], q.y * oss[kz]);
                    } else if constexpr (H16) {
                        const float2 q = __half22float2(oh[h][r]);
                        w = make_float2(q.x * os[h][r], q.y * os[h][r]);
                    } else {
                        w = obuf[p1(SPLIT * (j + R * r) + h, t)];
                    }
                    v[h][r] = MODE == COL_OTF ? cmul(v[h][r], w) : cmulc(v[h][r], w);
                }
                dft<R, +1>(v[h]);
            }
            // The refill below is a TMA (async-proxy) write over what every
            // thread just read through the generic proxy: each thread orders
            // its reads before it with a proxy fence, then the barrier.
            // Without the fence the refill could land under a slow warp's
            // reads when other kernels share the SM.
            if constexpr (OTF1) fence_proxy_async_smem();
            __syncthreads();
            if constexpr (OTF1) {
                // every thread has read the OTF buffer: refill it for the next tile
                if (tid == 0 && tile + (int)gridDim.x < total) issue_otf(tile + gridDim.x);
            }
#pragma unroll
            for (int h = 0; h < SPLIT; ++h)
#pragma unroll
                for (int r = 0; r < R; ++r) buf[p1(h * LH + j * R + r, t)] = v[h][r];
            __syncthreads();
#pragma unroll
            for (int h = 0; h < SPLIT; ++h) {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const float2 x = buf[p1(h * LH + j + R * r, t)];
                    v[h][r] = r == 0 ? x : cmulc(x, w2(r));
                }
                dft<R, +1>(v[h]);
            }
        }
        // ---- outputs in natural order ----
        if constexpr (MODE == COL_FWD) {
            // X[SPLIT m + h], m = j + R r
            if constexpr (SPLIT == 2) __syncthreads();  // other threads still read rows h LH + m
#pragma unroll
            for (int h = 0; h < SPLIT; ++h)
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int k = SPLIT * (j + R * r) + h;
                    if (k < a.nout) buf[p1(k, t)] = v[h][r];
                }
        } else {
            // y[n] = y0[n] (+ W_L^-n y1[n]), n = j + R r; this thread alone
            // read rows n and LH + n, so no barrier is needed before writing.
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int n = j + R * r;
                float2 y = v[0][r];
                if constexpr (SPLIT == 2) y = cadd(y, cmulc(v[1][r], ws(r)));
                if (n < a.nout) buf[p1(n, t)] = y;
            }
        }
        fence_proxy_async_smem();
        __syncthreads();
        if (tid == 0) {
            for (int r0 = 0; r0 < a.nout; r0 += a.dst_box) {
                if (a.dst_jdim == 1) tma_store_3d(&a.dst, c0, r0, o, buf + r0 * 16);
                else tma_store_3d(&a.dst, c0, o, r0, buf + r0 * 16);
            }
            tma_store_commit_and_wait();
            const int next = tile + NS * gridDim.x;
            if (next < total) issue(next, s);
        }
    }
}

}  // namespace dk
