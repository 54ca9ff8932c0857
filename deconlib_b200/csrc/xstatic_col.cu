// Instantiations of the plain-load column pass (colplain.cuh) at every
// static length, plus the runtime-radix form.
#include "colplain.cuh"

namespace dk {

void* pick_colfft_kernel(int L) {
#define DK_CASE(n) if (L == n) return (void*)k_colfft<n>;
    DK_STATIC_LENGTHS(DK_CASE)
#undef DK_CASE
    return (void*)k_colfft<0>;
}

}  // namespace dk
