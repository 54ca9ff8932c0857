// Instantiations of the X C2R pass (xpass.cuh): every epilogue at every
// static length, plus the runtime-radix form.
#include "xpass.cuh"

namespace dk {

template <int EPI>
static void* xc2r_for(int L) {
#define DK_CASE(n) if (L == n) return (void*)k_xc2r<EPI, n>;
    DK_STATIC_LENGTHS(DK_CASE)
#undef DK_CASE
    return (void*)k_xc2r<EPI, 0>;
}

void* pick_xc2r_kernel(int epi, int L) {
    switch (epi) {
        case EPI_STORE: return xc2r_for<EPI_STORE>(L);
        case EPI_RL_RATIO: return xc2r_for<EPI_RL_RATIO>(L);
        case EPI_RL_UPDATE: return xc2r_for<EPI_RL_UPDATE>(L);
        case EPI_PRED: return xc2r_for<EPI_PRED>(L);
        case EPI_DOWN2: return xc2r_for<EPI_DOWN2>(L);
        default: return nullptr;
    }
}

}  // namespace dk
