// Plain-load column pass (passes 2-4 for lengths without a TMA kernel):
// one CTA = T columns x L points of one plane, loaded with ordinary loads,
// transformed in shared memory (compile-time radices for the static
// lengths, the runtime-radix path otherwise), written back.
#pragma once

#include "conv_impl.cuh"

namespace dk {

template <int LS>
__global__ void __launch_bounds__(LS > 0 ? kFftThreads : kDynThreads, 1) k_colfft(ColArgs a) {
    extern __shared__ float2 sm[];
    const int T = a.T, L = a.ax.L, tid = threadIdx.x;
    const int64_t o = blockIdx.x / a.ntiles;
    const int64_t kx0 = (int64_t)(blockIdx.x - o * a.ntiles) * T;
    const float2* src = a.src + o * a.src_os + kx0;
    const int lgT = 31 - __clz(T);  // T is a power of two
    for (int q = tid; q < L * T; q += blockDim.x) {
        const int j = q >> lgT, t = q & (T - 1);
        float2 v = make_float2(0.f, 0.f);
        if (j < a.nin && kx0 + t < a.ncols) v = src[(int64_t)j * a.src_js + t];
        sm[phys(j, t, T)] = v;
    }
    __syncthreads();
    const int t = tid % T, jb = tid / T;
    if (a.mode == COL_INV) {
        fft_lines<+1, LS>(sm, T, t, jb, a.ax);
    } else {
        fft_lines<-1, LS>(sm, T, t, jb, a.ax);
    }
    if (a.mode == COL_OTF || a.mode == COL_OTF_CONJ) {
        const float2* otf = a.otf + o * a.otf_os + kx0;
        for (int q = tid; q < L * T; q += blockDim.x) {
            const int j = q >> lgT, tt = q & (T - 1);
            if (kx0 + tt < a.ncols) {
                const float2 w = __ldg(&otf[(int64_t)j * a.otf_js + tt]);
                const int p = phys(j, tt, T);
                sm[p] = a.mode == COL_OTF ? cmul(sm[p], w) : cmulc(sm[p], w);
            }
        }
        __syncthreads();
        fft_lines<+1, LS>(sm, T, t, jb, a.ax);
    }
    float2* dst = a.dst + o * a.dst_os + kx0;
    for (int q = tid; q < a.nout * T; q += blockDim.x) {
        const int j = q >> lgT, tt = q & (T - 1);
        if (kx0 + tt < a.ncols) dst[(int64_t)j * a.dst_js + tt] = sm[phys(j, tt, T)];
    }
}

}  // namespace dk
