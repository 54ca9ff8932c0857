// Deterministic FP64 reductions over float32 arrays.
//
// Pass 1 runs a grid whose size depends only on n; every CTA accumulates a
// grid-stride slice in double and writes one partial.  Pass 2 (one CTA) folds
// the partials in a fixed order.  The result is therefore bitwise identical
// from run to run, which the adaptive PDHG step-size branch relies on
// (pdhg_mlx.py:774-781 compares two reductions).
#include <cfloat>

#include "conv_impl.cuh"

namespace dk {

constexpr int kRedThreads = 256;
constexpr int kRedMaxBlocks = 1184;  // 8 per SM on a 148-SM B200

int64_t reduce_partials_needed() { return kRedMaxBlocks; }

static int red_blocks(int64_t n) {
    return (int)std::max<int64_t>(1, std::min<int64_t>(kRedMaxBlocks, cdiv(n, kRedThreads * 8)));
}

template <int OP>
__global__ void __launch_bounds__(kRedThreads) k_reduce1(const float* __restrict__ a,
                                                         const float* __restrict__ b, int64_t n,
                                                         double* __restrict__ partials) {
    double acc = OP == DECON_RED_MAX ? -DBL_MAX : 0.0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double va = (double)__ldg(a + i);
        if constexpr (OP == DECON_RED_SUM) acc += va;
        else if constexpr (OP == DECON_RED_SUMSQ) acc += va * va;
        else if constexpr (OP == DECON_RED_DIFFSQ) {
            const double d = va - (double)__ldg(b + i);
            acc += d * d;
        } else if constexpr (OP == DECON_RED_DOT) acc += va * (double)__ldg(b + i);
        else acc = fmax(acc, va);
    }
    if constexpr (OP == DECON_RED_MAX) {
        __shared__ double red[kRedThreads / 32];
        for (int o = 16; o > 0; o >>= 1) acc = fmax(acc, __shfl_down_sync(0xffffffffu, acc, o));
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
        __syncthreads();
        if (threadIdx.x == 0) {
            double m = red[0];
            for (int w = 1; w < kRedThreads / 32; ++w) m = fmax(m, red[w]);
            partials[blockIdx.x] = m;
        }
    } else {
        const double s = block_sum(acc);
        if (threadIdx.x == 0) partials[blockIdx.x] = s;
    }
}

template <bool MAX>
__global__ void __launch_bounds__(kRedThreads) k_reduce2(const double* __restrict__ partials, int n,
                                                         double* __restrict__ out) {
    double acc = MAX ? -DBL_MAX : 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc = MAX ? fmax(acc, partials[i]) : acc + partials[i];
    if (MAX) {
        __shared__ double red[kRedThreads / 32];
        for (int o = 16; o > 0; o >>= 1) acc = fmax(acc, __shfl_down_sync(0xffffffffu, acc, o));
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
        __syncthreads();
        if (threadIdx.x == 0) {
            double m = red[0];
            for (int w = 1; w < kRedThreads / 32; ++w) m = fmax(m, red[w]);
            *out = m;
        }
    } else {
        const double s = block_sum(acc);
        if (threadIdx.x == 0) *out = s;
    }
}

int reduce_f32(const float* a, const float* b, int64_t n, int op, double* out, double* partials,
               int64_t npartials, cudaStream_t st) {
    if (n <= 0) return fail(DECON_ERR_VALUE, "reduce: n must be positive");
    const int g = red_blocks(n);
    if (g > npartials) return fail(DECON_ERR_VALUE, "reduce: partials buffer too small");
    switch (op) {
        case DECON_RED_SUM: k_reduce1<DECON_RED_SUM><<<g, kRedThreads, 0, st>>>(a, b, n, partials); break;
        case DECON_RED_SUMSQ: k_reduce1<DECON_RED_SUMSQ><<<g, kRedThreads, 0, st>>>(a, b, n, partials); break;
        case DECON_RED_DIFFSQ: k_reduce1<DECON_RED_DIFFSQ><<<g, kRedThreads, 0, st>>>(a, b, n, partials); break;
        case DECON_RED_DOT: k_reduce1<DECON_RED_DOT><<<g, kRedThreads, 0, st>>>(a, b, n, partials); break;
        case DECON_RED_MAX: k_reduce1<DECON_RED_MAX><<<g, kRedThreads, 0, st>>>(a, b, n, partials); break;
        default: return fail(DECON_ERR_VALUE, "reduce: unknown op %d", op);
    }
    DK_LAUNCHED();
    if (op == DECON_RED_MAX) k_reduce2<true><<<1, kRedThreads, 0, st>>>(partials, g, out);
    else k_reduce2<false><<<1, kRedThreads, 0, st>>>(partials, g, out);
    DK_LAUNCHED();
    return DECON_OK;
}

int finish_partials(const double* partials, int n, double* out, cudaStream_t st) {
    k_reduce2<false><<<1, kRedThreads, 0, st>>>(partials, n, out);
    DK_LAUNCHED();
    return DECON_OK;
}

// max |z|^2 over a complex array with row pitch (OTF operator norm).
__global__ void __launch_bounds__(kRedThreads) k_maxabs2(const float2* __restrict__ z, int64_t rows,
                                                         int64_t cols, int64_t pitch,
                                                         double* __restrict__ partials) {
    double acc = 0.0;
    const int64_t n = rows * cols, stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const int64_t r = i / cols, c = i - r * cols;
        const float2 v = z[r * pitch + c];
        // |otf|^2 in float32, as the reference evaluates mx.abs(otf) ** 2
        const float m = sqrtf(v.x * v.x + v.y * v.y);
        acc = fmax(acc, (double)(m * m));
    }
    __shared__ double red[kRedThreads / 32];
    for (int o = 16; o > 0; o >>= 1) acc = fmax(acc, __shfl_down_sync(0xffffffffu, acc, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = red[0];
        for (int w = 1; w < kRedThreads / 32; ++w) m = fmax(m, red[w]);
        partials[blockIdx.x] = m;
    }
}

int max_abs2(const float2* z, int64_t rows, int64_t cols, int64_t pitch, double* out,
             double* partials, cudaStream_t st) {
    const int g = red_blocks(rows * cols);
    k_maxabs2<<<g, kRedThreads, 0, st>>>(z, rows, cols, pitch, partials);
    DK_LAUNCHED();
    k_reduce2<true><<<1, kRedThreads, 0, st>>>(partials, g, out);
    DK_LAUNCHED();
    return DECON_OK;
}

}  // namespace dk

extern "C" int64_t decon_reduce_workspace_bytes(void) {
    return dk::reduce_partials_needed() * (int64_t)sizeof(double);
}

extern "C" int decon_reduce(const float* a, const float* b, int64_t n, int op, double* out,
                            void* workspace, void* stream) {
    using namespace dk;
    if (!a || !out || !workspace || ((op == DECON_RED_DIFFSQ || op == DECON_RED_DOT) && !b))
        return fail(DECON_ERR_NULL, "decon_reduce: null pointer");
    return reduce_f32(a, b, n, op, out, static_cast<double*>(workspace), reduce_partials_needed(),
                      as_stream(stream));
}
