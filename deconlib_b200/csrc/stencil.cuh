// Hessian3D stencil arithmetic shared by the stand-alone operator kernels
// (ops.cu) and the fused PDHG kernels (solvers.cu), so both produce the same
// float32 values.  Neumann boundaries by index clamping, operation order as in
// deconlib's linops_core_mlx.py:25-80 and linops_mlx.py:224-259.
#pragma once

#include "common.cuh"

namespace dk {

__device__ __forceinline__ int64_t clampi(int64_t v, int64_t n) { return v < 0 ? 0 : (v >= n ? n - 1 : v); }

// d2 along one axis (linops_core_mlx.py:66-76): (f[i-1] - 2 f[i]) + f[i+1].
// The stencil arithmetic uses round-to-nearest intrinsics throughout: every
// product and sum is rounded as the reference's float32 array operations
// round it, and no multiply-add is contracted, so every kernel that inlines
// these functions (fused or not) produces the same bits.
__device__ __forceinline__ float d2v(float fm, float f0, float fp) {
    return __fadd_rn(__fsub_rn(fm, __fmul_rn(2.f, f0)), fp);
}
// w * v rounded (a weighted component value)
__device__ __forceinline__ float wmul(float v, float w) { return __fmul_rn(v, w); }
// The element-wise PDHG updates, each operation rounded as the reference's
// float32 arrays round it (pdhg_mlx.py:724, 733, 742, 841):
//   x_bar = x + theta (x - x_prev), dual argument y + sigma K x_bar,
//   x_new = max(0, x - tau g)
__device__ __forceinline__ float xbar_of(float x, float xp, float th) {
    return __fadd_rn(x, __fmul_rn(th, __fsub_rn(x, xp)));
}
__device__ __forceinline__ float dual_arg(float y, float sg, float kx) {
    return __fadd_rn(y, __fmul_rn(sg, kx));
}
__device__ __forceinline__ float primal_of(float x, float tau, float g) {
    return fmaxf(__fsub_rn(x, __fmul_rn(tau, g)), 0.f);
}

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
    return j < 0 ? -wmul(__ldg(g), w) : (j >= n ? -wmul(__ldg(g + (n - 1) * s), w) : wmul(__ldg(g + j * s), w));
}

__device__ __forceinline__ float inner_adj(const float* g, int64_t ia, int64_t na, int64_t sa,
                                           float w) {
    return __fsub_rn(gext(g, ia - 1, na, sa, w), gext(g, ia + 1, na, sa, w)) / 2.f;
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
    return __fsub_rn(row(ib - 1), row(ib + 1)) / 2.f;
}

// d2 of a weighted component h * w along one axis with edge replication.
__device__ __forceinline__ float d2w(const float* g, int64_t i, int64_t n, int64_t s, float w) {
    const float fm = wmul(__ldg(g + clampi(i - 1, n) * s), w);
    const float f0 = wmul(__ldg(g + i * s), w);
    const float fp = wmul(__ldg(g + clampi(i + 1, n) * s), w);
    return d2v(fm, f0, fp);
}

// Hessian3D.adjoint at voxel (z, y, x) (linops_mlx.py:244-259) for any
// accessor G(c, z, y, x) -> component c at in-range coordinates: the six
// adjoint stencils (weights applied per element, boundary sign flips of
// d1_cen_adj) summed in the reference's order.  The global-memory and the
// shared-memory tiled kernels both use this one definition.
template <class G>
__device__ __forceinline__ float hess_adj_gen(const G& g, int64_t z, int64_t y, int64_t x,
                                              const Dims& d, const float w[6]) {
    // d2 of the weighted component c along one axis, edge-replicated
    const float azz = d2v(wmul(g(0, clampi(z - 1, d.nz), y, x), w[0]), wmul(g(0, z, y, x), w[0]),
                          wmul(g(0, clampi(z + 1, d.nz), y, x), w[0]));
    const float ayy = d2v(wmul(g(1, z, clampi(y - 1, d.ny), x), w[1]), wmul(g(1, z, y, x), w[1]),
                          wmul(g(1, z, clampi(y + 1, d.ny), x), w[1]));
    const float axx = d2v(wmul(g(2, z, y, clampi(x - 1, d.nx)), w[2]), wmul(g(2, z, y, x), w[2]),
                          wmul(g(2, z, y, clampi(x + 1, d.nx)), w[2]));
    // d1_cen_adj(d1_cen_adj(., inner axis), outer axis); G(-1) = -g[0], G(n) = -g[n-1]
    auto ext = [&](int c, int64_t zz, int64_t yy, int64_t xx, int axis, float wc) -> float {
        int64_t n = axis == 0 ? d.nz : (axis == 1 ? d.ny : d.nx);
        int64_t v = axis == 0 ? zz : (axis == 1 ? yy : xx);
        const bool neg = v < 0 || v >= n;
        const int64_t cl = v < 0 ? 0 : (v >= n ? n - 1 : v);
        if (axis == 0) zz = cl;
        else if (axis == 1) yy = cl;
        else xx = cl;
        const float val = wmul(g(c, zz, yy, xx), wc);
        return neg ? -val : val;
    };
    // inner adjoint along axis a at outer index ob (axis b), evaluated at point p
    auto inner = [&](int c, int b, int64_t ob, int a, int64_t z0, int64_t y0, int64_t x0,
                     float wc) -> float {
        int64_t zz = z0, yy = y0, xx = x0;
        if (b == 0) zz = ob;
        else if (b == 1) yy = ob;
        else xx = ob;
        int64_t zm = zz, ym = yy, xm = xx, zp = zz, yp = yy, xp = xx;
        if (a == 0) { zm -= 1; zp += 1; }
        else if (a == 1) { ym -= 1; yp += 1; }
        else { xm -= 1; xp += 1; }
        return __fsub_rn(ext(c, zm, ym, xm, a, wc), ext(c, zp, yp, xp, a, wc)) / 2.f;
    };
    auto mixed = [&](int c, int b, int a, float wc) -> float {
        const int64_t nb = b == 0 ? d.nz : (b == 1 ? d.ny : d.nx);
        const int64_t ib = b == 0 ? z : (b == 1 ? y : x);
        auto row = [&](int64_t jb) -> float {
            if (jb < 0) return -inner(c, b, 0, a, z, y, x, wc);
            if (jb >= nb) return -inner(c, b, nb - 1, a, z, y, x, wc);
            return inner(c, b, jb, a, z, y, x, wc);
        };
        return __fsub_rn(row(ib - 1), row(ib + 1)) / 2.f;
    };
    const float ayz = mixed(3, 0, 1, w[3]);
    const float axz = mixed(4, 0, 2, w[4]);
    const float axy = mixed(5, 1, 2, w[5]);
    return __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(azz, ayy), axx), ayz), axz), axy);
}

// Accessor of the six components stored as hw[c * n + i].
struct Hess6Global {
    const float* hw;
    int64_t n, ny, nx;
    __device__ __forceinline__ float operator()(int c, int64_t z, int64_t y, int64_t x) const {
        return __ldg(hw + c * n + (z * ny + y) * nx + x);
    }
};

__device__ __forceinline__ float hess_adj_at(const float* hw, int64_t z, int64_t y, int64_t x,
                                             const Dims& d, const float w[6]) {
    const Hess6Global g{hw, d.nz * d.ny * d.nx, d.ny, d.nx};
    return hess_adj_gen(g, z, y, x, d, w);
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

// Hessian3D.adjoint of six stored components hw[c * n + i] on the tiled,
// staged walk of the fused PDHG kernels (solvers.cu).
int hess_adjoint_tiled(const float* hw, float* out, const Dims& d, const W6& w, cudaStream_t st);

}  // namespace dk
