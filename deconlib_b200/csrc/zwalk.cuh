// Tile geometry of the fused Hessian stencils and the register z-walk that
// evaluates Hessian3D of one or more fields over a CTA's tiles.
//
// A CTA of 32 x 8 threads owns an (x, y) tile and marches along z through a
// chunk of kZChunk planes; CTAs walk a fixed list of tiles (tile b, b + grid,
// ...), so per-CTA sums are deterministic.
#pragma once

#include "stencil.cuh"

namespace dk {

constexpr int kTX = 32, kTY = 8, kHX = kTX + 2, kHY = kTY + 2, kPL = kHX * kHY;
constexpr int kZChunk = 16;

struct TileGeo {
    int64_t ntx, nty, ntz, ntiles;
    __host__ __device__ TileGeo(const Dims& d)
        : ntx((d.nx + kTX - 1) / kTX), nty((d.ny + kTY - 1) / kTY),
          ntz((d.nz + kZChunk - 1) / kZChunk), ntiles(0) {
        ntiles = ntx * nty * ntz;
    }
};

__device__ __forceinline__ int sidx(int64_t yy, int64_t xx, int64_t y0, int64_t x0) {
    return (int)((yy - y0 + 1) * kHX + (xx - x0 + 1));
}

// This thread's (up to two) halo-plane elements: fixed (row, column) of the
// staged tile, loaded into registers one plane ahead of use.
struct StageSlots {
    int q[2];
    int64_t off[2];  // in-plane offset (clamped y, x)
    bool ok[2];
    __device__ __forceinline__ StageSlots(int64_t x0, int64_t y0, const Dims& d) {
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            q[u] = threadIdx.x + u * blockDim.x;
            ok[u] = q[u] < kPL;
            const int ly = q[u] / kHX, lx = q[u] - ly * kHX;
            off[u] = clampi(y0 - 1 + ly, d.ny) * d.nx + clampi(x0 - 1 + lx, d.nx);
        }
    }
    // f(plane_offset + in_plane_offset) for plane zz
    template <class F>
    __device__ __forceinline__ void load(float r[2], const F& f, int64_t zz, int64_t plane) const {
#pragma unroll
        for (int u = 0; u < 2; ++u) r[u] = ok[u] ? f(zz * plane + off[u]) : 0.f;
    }
    __device__ __forceinline__ void store(float* p, const float r[2]) const {
#pragma unroll
        for (int u = 0; u < 2; ++u)
            if (ok[u]) p[q[u]] = r[u];
    }
};

// Hessian3D of NF fields over this CTA's tiles with the z axis walked in
// registers.  Each thread owns (up to two) positions of the 34 x 10 tile +
// halo plane and keeps every field at z - 1, z, z + 1 of them in registers
// (the raw loads of the next plane in flight one plane ahead); per plane it
// publishes the three values its neighbours' stencils take from it: the
// field, the half central z-difference (f(z+1) - f(z-1)) / 2 and the second
// z-difference.  Planes are double-buffered, so a plane costs one CTA
// barrier.  Every float operation is hess6_smem's (hess6 of stencil.cuh),
// evaluated by the owner of an operand instead of its reader, so the
// components are bit-identical to the operator's.
//   raw(i)       -> RawT: the loads behind the fields at linear index i
//   val(r, k)    -> float: field k from them
//   body(i, h)   voxel i of the tile interior, h[k][0..6) the weighted
//                components of field k
// IDX is the type of element offsets (uint32_t when every offset the
// kernel forms fits 32 bits, which the launchers check with
// offsets_fit_u32, else int64_t); per-tile quantities are set once per
// tile and plane offsets advance by additions, since the walk is bound by
// instruction issue.
template <class IDX, int NF, class Raw, class Val, class Body>
__device__ __forceinline__ void hess_zwalk(const Dims& d, const W6& w, const Raw& raw, const Val& val,
                                           const Body& body) {
    using RawT = decltype(raw(IDX(0)));
    __shared__ float sp[2][NF][kPL], sh[2][NF][kPL], sz[2][NF][kPL];
    const IDX plane = (IDX)(d.ny * d.nx);
    const int nz = (int)d.nz;
    const TileGeo g(d);
    const int tid = threadIdx.x, tx = tid % kTX, ty = tid / kTX;
    const int c = (ty + 1) * kHX + (tx + 1);
    const int n = c - kHX, so = c + kHX, wv = c - 1, e = c + 1;
    // this thread's two halo-window slots (the second exists for tid < kPL - 256)
    const int q1 = tid + 256;
    const bool ok1 = q1 < kPL;
    const int ly0 = tid / kHX, lx0 = tid - ly0 * kHX, ly1 = q1 / kHX, lx1 = q1 - ly1 * kHX;
    int buf = 0;
    for (int64_t tile = blockIdx.x; tile < g.ntiles; tile += gridDim.x) {
        const int64_t bx = tile % g.ntx, r = tile / g.ntx, by = r % g.nty, bz = r / g.nty;
        const int64_t x0 = bx * kTX, y0 = by * kTY;
        const int z0 = (int)(bz * kZChunk);
        const int z1 = z0 + kZChunk < nz ? z0 + kZChunk : nz;
        const bool in = x0 + tx < d.nx && y0 + ty < d.ny;
        const IDX ipl = in ? (IDX)((y0 + ty) * d.nx + (x0 + tx)) : (IDX)0;
        const IDX off[2] = {(IDX)(clampi(y0 - 1 + ly0, d.ny) * d.nx + clampi(x0 - 1 + lx0, d.nx)),
                            ok1 ? (IDX)(clampi(y0 - 1 + ly1, d.ny) * d.nx + clampi(x0 - 1 + lx1, d.nx)) : (IDX)0};
        const int q[2] = {tid, q1};
        const bool ok[2] = {true, ok1};
        float vm[2][NF], vc[2][NF];
        RawT rq[2];
        IDX zo = (IDX)z0 * plane;  // offset of plane z
        {
            const IDX zb = (IDX)(z0 > 0 ? z0 - 1 : 0) * plane, zq = (IDX)(z0 + 1 < nz ? z0 + 1 : nz - 1) * plane;
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                if (ok[u]) {
                    const RawT a = raw(zb + off[u]), b = raw(zo + off[u]);
#pragma unroll
                    for (int k = 0; k < NF; ++k) {
                        vm[u][k] = val(a, k);
                        vc[u][k] = val(b, k);
                    }
                    rq[u] = raw(zq + off[u]);
                } else {
#pragma unroll
                    for (int k = 0; k < NF; ++k) vm[u][k] = vc[u][k] = 0.f;
                    rq[u] = RawT{};
                }
            }
        }
        for (int z = z0; z < z1; ++z) {
            float vp[2][NF];
            const IDX zi = zo;  // plane z
            zo += plane;        // plane z + 1
            const IDX zq = z + 2 < nz ? zo + plane : zo;  // clamp(z + 2)
#pragma unroll
            for (int u = 0; u < 2; ++u) {
#pragma unroll
                for (int k = 0; k < NF; ++k) vp[u][k] = val(rq[u], k);
                if (ok[u] && z + 1 < z1) rq[u] = raw(zq + off[u]);
                if (ok[u]) {
#pragma unroll
                    for (int k = 0; k < NF; ++k) {
                        sp[buf][k][q[u]] = vc[u][k];
                        sh[buf][k][q[u]] = (vp[u][k] - vm[u][k]) / 2.f;
                        sz[buf][k][q[u]] = d2v(vm[u][k], vc[u][k], vp[u][k]);
                    }
                }
            }
            __syncthreads();
            if (in) {
                float h[NF][6];
#pragma unroll
                for (int k = 0; k < NF; ++k) {
                    const float* P = sp[buf][k];
                    const float* Hz = sh[buf][k];
                    const float cv = P[c];
                    h[k][0] = sz[buf][k][c] * w.w[0];
                    h[k][1] = d2v(P[n], cv, P[so]) * w.w[1];
                    h[k][2] = d2v(P[wv], cv, P[e]) * w.w[2];
                    h[k][3] = ((Hz[so] - Hz[n]) / 2.f) * w.w[3];
                    h[k][4] = ((Hz[e] - Hz[wv]) / 2.f) * w.w[4];
                    const float dy_xp = (P[so + 1] - P[n + 1]) / 2.f;
                    const float dy_xm = (P[so - 1] - P[n - 1]) / 2.f;
                    h[k][5] = ((dy_xp - dy_xm) / 2.f) * w.w[5];
                }
                body(zi + ipl, h);
            }
            buf ^= 1;
#pragma unroll
            for (int u = 0; u < 2; ++u)
#pragma unroll
                for (int k = 0; k < NF; ++k) {
                    vm[u][k] = vc[u][k];
                    vc[u][k] = vp[u][k];
                }
        }
    }
}

// Element offsets fit 32 bits when all six components of a Hessian do.
inline bool offsets_fit_u32(const Dims& d) { return 6 * d.nz * d.ny * d.nx < (int64_t(1) << 32); }

}  // namespace dk
