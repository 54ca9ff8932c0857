// Instantiations of the X R2C pass (xpass.cuh): every prologue at every
// static length, plus the runtime-radix form.
#include "xpass.cuh"

namespace dk {

template <int PRO>
static void* xr2c_for(int L) {
#define DK_CASE(n) if (L == n) return (void*)k_xr2c<PRO, n>;
    DK_STATIC_LENGTHS(DK_CASE)
#undef DK_CASE
    return (void*)k_xr2c<PRO, 0>;
}

void* pick_xr2c_kernel(int pro, int L) {
    switch (pro) {
        case PRO_ARRAY: return xr2c_for<PRO_ARRAY>(L);
        case PRO_CONST: return xr2c_for<PRO_CONST>(L);
        case PRO_KERNEL: return xr2c_for<PRO_KERNEL>(L);
        case PRO_RLINIT: return xr2c_for<PRO_RLINIT>(L);
        case PRO_UP2: return xr2c_for<PRO_UP2>(L);
        default: return nullptr;
    }
}

}  // namespace dk
