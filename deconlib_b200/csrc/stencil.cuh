// Hessian3D stencil arithmetic shared by the stand-alone operator kernels
// (ops.cu) and the fused PDHG kernels (solvers.cu), so both produce the same
// float32 values.  Neumann boundaries by index clamping, operation order as in
// deconlib's linops_core_mlx.py:25-80 and linops_mlx.py:224-259.
#pragma once

#include "common.cuh"

namespace dk {

__device__ __forceinline__ int64_t clampi(int64_t v, int64_t n) { return v < 0 ? 0 : (v >= n ? n - 1 : v); }

// d2 along one axis (linops_core_mlx.py:66-76): (f[i-1] - 2 f[i]) + f[i+1].
__device__ __forceinline__ float d2v(float fm, float f0, float fp) { return fm - 2.f * f0 + fp; }

struct Dims {
    int64_t nz, ny, nx;
};

// Weighted Hessian [zz, yy, xx, yz, xz, xy] at (z, y, x) of the field f(z, y, x)
// (linops_mlx.py:224-242; d1_cen of d1_cen for the mixed terms).
template <class F>
__device__ __forceinline__ void hess6(const F& f, int64_t z, int64_t y, int64_t x, const Dims& d,
                                      const float w[6], float h[6]) {
    const int64_t zm = clampi(z - 1, d.nz), zp = clampi(z + 1, d.nz);
    const int64_t ym = clampi(y - 1, d.ny), yp = clampi(y + 1, d.ny);
    const int64_t xm = clampi(x - 1, d.nx), xp = clampi(x + 1, d.nx);
    const float c = f(z, y, x);
    const float hzz = d2v(f(zm, y, x), c, f(zp, y, x));
    const float hyy = d2v(f(z, ym, x), c, f(z, yp, x));
    const float hxx = d2v(f(z, y, xm), c, f(z, y, xp));
    const float dz_yp = (f(zp, yp, x) - f(zm, yp, x)) / 2.f;
    const float dz_ym = (f(zp, ym, x) - f(zm, ym, x)) / 2.f;
    const float hyz = (dz_yp - dz_ym) / 2.f;
    const float dz_xp = (f(zp, y, xp) - f(zm, y, xp)) / 2.f;
    const float dz_xm = (f(zp, y, xm) - f(zm, y, xm)) / 2.f;
    const float hxz = (dz_xp - dz_xm) / 2.f;
    const float dy_xp = (f(z, yp, xp) - f(z, ym, xp)) / 2.f;
    const float dy_xm = (f(z, yp, xm) - f(z, ym, xm)) / 2.f;
    const float hxy = (dy_xp - dy_xm) / 2.f;
    h[0] = hzz * w[0];
    h[1] = hyy * w[1];
    h[2] = hxx * w[2];
    h[3] = hyz * w[3];
    h[4] = hxz * w[4];
    h[5] = hxy * w[5];
}

// d1_cen_adj (linops_core_mlx.py:53-58): out[i] = (G(i-1) - G(i+1)) / 2 with
// G(-1) = -g[0], G(n) = -g[n-1].  Each element is first multiplied by its
// component weight (H_w = H * w, linops_mlx.py:250), the float32 product the
// reference forms.
__device__ __forceinline__ float gext(const float* g, int64_t j, int64_t n, int64_t s, float w) {
    return j < 0 ? -(__ldg(g) * w) : (j >= n ? -(__ldg(g + (n - 1) * s) * w) : __ldg(g + j * s) * w);
}

__device__ __forceinline__ float inner_adj(const float* g, int64_t ia, int64_t na, int64_t sa,
                                           float w) {
    return (gext(g, ia - 1, na, sa, w) - gext(g, ia + 1, na, sa, w)) / 2.f;
}

// d1_cen_adj along axis b of (d1_cen_adj along axis a of H) at (ib, ia) of a
// 2-D slice g (strides sb, sa): inner adjoint at ib -+ 1, then the outer one.
__device__ __forceinline__ float mixed_adj(const float* g, int64_t ib, int64_t nb, int64_t sb,
                                           int64_t ia, int64_t na, int64_t sa, float w) {
    auto row = [&](int64_t jb) -> float {
        if (jb < 0) return -inner_adj(g, ia, na, sa, w);
        if (jb >= nb) return -inner_adj(g + (nb - 1) * sb, ia, na, sa, w);
        return inner_adj(g + jb * sb, ia, na, sa, w);
    };
    return (row(ib - 1) - row(ib + 1)) / 2.f;
}

// d2 of a weighted component h * w along one axis with edge replication.
__device__ __forceinline__ float d2w(const float* g, int64_t i, int64_t n, int64_t s, float w) {
    const float fm = __ldg(g + clampi(i - 1, n) * s) * w;
    const float f0 = __ldg(g + i * s) * w;
    const float fp = __ldg(g + clampi(i + 1, n) * s) * w;
    return d2v(fm, f0, fp);
}

// Hessian3D.adjoint at voxel (z, y, x) of the six components hw[c * n + i]
// (linops_mlx.py:244-259): the six adjoint stencils summed in the reference's order.
__device__ __forceinline__ float hess_adj_at(const float* hw, int64_t z, int64_t y, int64_t x,
                                             const Dims& d, const float w[6]) {
    const int64_t n = d.nz * d.ny * d.nx;
    const int64_t sz = d.ny * d.nx, sy = d.nx, sx = 1;
    const float azz = d2w(hw + y * sy + x, z, d.nz, sz, w[0]);
    const float ayy = d2w(hw + n + z * sz + x, y, d.ny, sy, w[1]);
    const float axx = d2w(hw + 2 * n + z * sz + y * sy, x, d.nx, sx, w[2]);
    const float ayz = mixed_adj(hw + 3 * n + x, z, d.nz, sz, y, d.ny, sy, w[3]);
    const float axz = mixed_adj(hw + 4 * n + y * sy, z, d.nz, sz, x, d.nx, sx, w[4]);
    const float axy = mixed_adj(hw + 5 * n + z * sz, y, d.ny, sy, x, d.nx, sx, w[5]);
    return ((((azz + ayy) + axx) + ayz) + axz) + axy;
}

// Component weights [r^2, 1, 1, sqrt2 r, sqrt2 r, sqrt2] (linops_mlx.py:237-239;
// SQRT2 is a float32 device scalar there).
inline void hessian_weights(float r, float w[6]) {
    const float s2 = sqrtf(2.f);
    w[0] = (float)((double)r * (double)r);
    w[1] = 1.f;
    w[2] = 1.f;
    w[3] = r * s2;
    w[4] = r * s2;
    w[5] = s2;
}

struct W6 {
    float w[6];
};

}  // namespace dk
