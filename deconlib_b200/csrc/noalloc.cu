// decon_reduce_noalloc: the FP64 reduction of decon_reduce for callers that
// cannot allocate device memory.
//
// Who needs it: code that runs where cudaMalloc is not an option, for example
// a plug-in inside a host application that owns every device allocation, or a
// latency-critical pipeline whose memory is reserved up front because
// cudaMalloc can synchronise the device and can fail at run time.  Such
// callers own their inputs and the output double but cannot provide the
// workspace decon_reduce asks for.
//
// How: the per-block partial sums live in the file-scope device array below
// (kNoAllocSlots doubles = 128 KB, held by every GPU that loads the library
// until the process exits).  Pass 1 gives each block one fixed chunk of
// kNoAllocChunk elements, so n is limited to kNoAllocSlots * kNoAllocChunk
// elements; pass 2 folds the partials in fixed order (deterministic).  Host
// code cannot pass the array's name to a kernel (it is a host-side stand-in,
// not a device address): the first call on each device (in each CUDA context
// of that device), with that device current, looks the address up with
// cudaGetSymbolAddress and keeps it.
#include <cuda.h>

#include <mutex>

#include "conv_impl.cuh"

namespace dk {

constexpr int kNoAllocThreads = 256;
constexpr int64_t kNoAllocChunk = 4096;  // elements per block in pass 1
constexpr int kNoAllocSlots = 16384;     // partial sums (128 KB)
constexpr int64_t kNoAllocMaxN = kNoAllocChunk * kNoAllocSlots;

static __device__ __align__(256) double g_noalloc_partials[kNoAllocSlots];

template <int OP>
__device__ __forceinline__ double red_elem(const float* a, const float* b, int64_t i) {
    const double va = (double)__ldg(a + i);
    if constexpr (OP == DECON_RED_SUM) return va;
    else if constexpr (OP == DECON_RED_SUMSQ) return va * va;
    else if constexpr (OP == DECON_RED_DIFFSQ) {
        const double d = va - (double)__ldg(b + i);
        return d * d;
    } else if constexpr (OP == DECON_RED_DOT) return va * (double)__ldg(b + i);
    else return va;  // MAX
}

template <int OP>
__global__ void __launch_bounds__(kNoAllocThreads) k_na_pass1(const float* __restrict__ a,
                                                              const float* __restrict__ b,
                                                              int64_t n, double* partials) {
    const int64_t lo = (int64_t)blockIdx.x * kNoAllocChunk;
    const int64_t hi = min(n, lo + kNoAllocChunk);
    double acc = OP == DECON_RED_MAX ? -1.0e308 : 0.0;
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const double v = red_elem<OP>(a, b, i);
        acc = OP == DECON_RED_MAX ? fmax(acc, v) : acc + v;
    }
    __shared__ double red[kNoAllocThreads / 32];
    if constexpr (OP == DECON_RED_MAX) {
        for (int o = 16; o > 0; o >>= 1) acc = fmax(acc, __shfl_down_sync(0xffffffffu, acc, o));
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
        __syncthreads();
        if (threadIdx.x == 0) {
            double m = red[0];
            for (int w = 1; w < kNoAllocThreads / 32; ++w) m = fmax(m, red[w]);
            partials[blockIdx.x] = m;
        }
    } else {
        const double s = block_sum(acc);
        if (threadIdx.x == 0) partials[blockIdx.x] = s;
    }
}

template <bool MAX>
__global__ void __launch_bounds__(kNoAllocThreads) k_na_pass2(const double* partials, int nb,
                                                              double* out) {
    double acc = MAX ? -1.0e308 : 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) acc = MAX ? fmax(acc, partials[i]) : acc + partials[i];
    __shared__ double red[kNoAllocThreads / 32];
    if (MAX) {
        for (int o = 16; o > 0; o >>= 1) acc = fmax(acc, __shfl_down_sync(0xffffffffu, acc, o));
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
        __syncthreads();
        if (threadIdx.x == 0) {
            double m = red[0];
            for (int w = 1; w < kNoAllocThreads / 32; ++w) m = fmax(m, red[w]);
            *out = m;
        }
    } else {
        const double s = block_sum(acc);
        if (threadIdx.x == 0) *out = s;
    }
}

// Device address of g_noalloc_partials.  The address belongs to the module
// as loaded into one CUDA context, so it is cached per device together with
// the id of the context it was looked up in (cuCtxGetId, unique for the life
// of the process) and looked up again when the device's current context is
// another one (after cudaDeviceReset, or a primary context released and
// created again).  Without the driver's context queries it is looked up on
// every call.
using PfnCtxGetCurrent = CUresult (*)(CUcontext*);
using PfnCtxGetId = CUresult (*)(CUcontext, unsigned long long*);

static bool current_context_id(unsigned long long* id) {
    static PfnCtxGetCurrent get_current = nullptr;
    static PfnCtxGetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<PfnCtxGetCurrent>(fn);
        else
            cudaGetLastError();
        fn = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<PfnCtxGetId>(fn);
        else
            cudaGetLastError();
    });
    if (!get_current || !get_id) return false;
    CUcontext c = nullptr;
    if (get_current(&c) != CUDA_SUCCESS || c == nullptr) return false;
    return get_id(c, id) == CUDA_SUCCESS;
}

static int noalloc_scratch(double** out) {
    static std::mutex mu;
    static double* addr[64] = {nullptr};
    static unsigned long long ctx[64] = {0};
    int dev = 0;
    DK_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(DECON_ERR_UNSUPPORTED, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(mu);
    unsigned long long id = 0;
    bool have_id = current_context_id(&id);
    if (have_id && addr[dev] && ctx[dev] == id) {
        *out = addr[dev];
        return DECON_OK;
    }
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess || p == nullptr)
        return fail(DECON_ERR_CUDA, "cudaGetSymbolAddress of the no-alloc scratch failed: %s",
                    cudaGetErrorString(e));
    // the lookup makes the device's primary context current if none was
    if (!have_id) have_id = current_context_id(&id);
    addr[dev] = have_id ? static_cast<double*>(p) : nullptr;  // no id: look up on every call
    ctx[dev] = have_id ? id : 0;
    *out = static_cast<double*>(p);
    return DECON_OK;
}

}  // namespace dk

// See include/decon_b200.h.  No cudaMalloc / cudaFree / allocating library
// call happens here or in the kernels.  Every call shares the one scratch
// array, which keeps the previous call's partial sums: pass 1 overwrites each
// partial it uses before pass 2 reads it, so nothing needs clearing, but two
// calls whose kernels overlap on the GPU (different streams, no ordering)
// race on the array.
extern "C" int decon_reduce_noalloc(const float* a, const float* b, int64_t n, int op, double* out,
                                    void* stream) {
    using namespace dk;
    if (!a || !out || ((op == DECON_RED_DIFFSQ || op == DECON_RED_DOT) && !b))
        return fail(DECON_ERR_NULL, "decon_reduce_noalloc: null pointer");
    if (n <= 0) return fail(DECON_ERR_VALUE, "decon_reduce_noalloc: n must be positive");
    if (n > kNoAllocMaxN)
        return fail(DECON_ERR_VALUE,
                    "decon_reduce_noalloc: n = %lld exceeds the fixed scratch capacity of %lld "
                    "elements (use decon_reduce with a workspace)",
                    (long long)n, (long long)kNoAllocMaxN);
    double* partials = nullptr;
    DK_TRY(noalloc_scratch(&partials));
    const cudaStream_t st = as_stream(stream);
    const int nb = (int)cdiv(n, kNoAllocChunk);
    switch (op) {
        case DECON_RED_SUM: k_na_pass1<DECON_RED_SUM><<<nb, kNoAllocThreads, 0, st>>>(a, b, n, partials); break;
        case DECON_RED_SUMSQ: k_na_pass1<DECON_RED_SUMSQ><<<nb, kNoAllocThreads, 0, st>>>(a, b, n, partials); break;
        case DECON_RED_DIFFSQ: k_na_pass1<DECON_RED_DIFFSQ><<<nb, kNoAllocThreads, 0, st>>>(a, b, n, partials); break;
        case DECON_RED_DOT: k_na_pass1<DECON_RED_DOT><<<nb, kNoAllocThreads, 0, st>>>(a, b, n, partials); break;
        case DECON_RED_MAX: k_na_pass1<DECON_RED_MAX><<<nb, kNoAllocThreads, 0, st>>>(a, b, n, partials); break;
        default: return fail(DECON_ERR_VALUE, "decon_reduce_noalloc: unknown op %d", op);
    }
    DK_LAUNCHED();
    if (op == DECON_RED_MAX) k_na_pass2<true><<<1, kNoAllocThreads, 0, st>>>(partials, nb, out);
    else k_na_pass2<false><<<1, kNoAllocThreads, 0, st>>>(partials, nb, out);
    DK_LAUNCHED();
    return DECON_OK;
}
