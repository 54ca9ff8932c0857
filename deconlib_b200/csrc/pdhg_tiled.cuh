// Shared-memory tiled, software-pipelined forms of the fused Hessian-PDHG
// kernels.
//
// A CTA of 32 x 8 threads owns an (x, y) tile and marches along z through a
// chunk of kZChunk planes; CTAs walk a fixed list of tiles (tile b, b + grid,
// ...) so the FP64 partial sums are per-CTA and deterministic.  The planes
// of every field the stencil reads (with a one-voxel halo) and the
// centre-only operands stream into shared memory with 4-byte cp.async, D
// planes ahead of use, as one continuous stream across the CTA's tiles: the
// loads never wait on the arithmetic and the arithmetic waits on a load only
// when the D-deep pipeline runs dry.  Each thread consumes exactly the
// elements it copied (its own cp.async group), converts them into a 4-plane
// working ring (e.g. x_bar = x + theta (x - x_prev)), and one barrier per
// plane makes the ring visible to the CTA; the 4th ring plane lets a plane be
// written while slower threads still read the previous three.  The
// arithmetic is the shared stencil code with shared-memory accessors, so the
// results equal the untiled kernels bit for bit.
//
// The primal update (k_hess_primal_t: six staged y2 components, x and
// A^T y1) keeps a one-plane register prefetch and static three-plane rings
// (hess_adj_walk, shared with the standalone Hessian3D adjoint).  It is
// bound by instruction issue, so the walk indexes with 32-bit element
// offsets and sets everything per tile once: 64 registers, four CTAs per SM
// (on the B200 92 us at 128x256x256 against 131 us for the same walk with
// 64-bit indexing at 122 registers, and against 141-150 us for a form that
// staged the operands by TMA through an mbarrier ring).  The pipelined
// cp.async form measured slower too (six deep rings cost occupancy and
// issue slots).
//
// ||H (x_new - x)||^2 (k_hess_dk_r) walks z in registers instead
// (hess_zwalk): each thread keeps three planes of its halo positions and
// publishes per plane only what its neighbours' stencils need; on the B200
// this cut the launch's instruction count and the PDHG iteration by ~1.5 %
// against the pipelined form.  The same walk for the dual update measured no
// faster than k_hess_dual_p and is not used there.
#pragma once

#include "solvers.cuh"
#include "stencil.cuh"
#include "zwalk.cuh"

namespace dk {

// Hessian components at tile-local (ly, lx) (1-based, halo at 0 and kT+1)
// from staged planes: clamping is already in the staged values, so the taps
// are plain neighbours; the float ops are those of hess6.
__device__ __forceinline__ void hess6_smem(const float* pm, const float* p0, const float* pp, int ly,
                                           int lx, const float w[6], float h[6]) {
    const int c = ly * kHX + lx;
    const int n = c - kHX, s = c + kHX, wv = c - 1, e = c + 1;
    const float cv = p0[c];
    const float hzz = d2v(pm[c], cv, pp[c]);
    const float hyy = d2v(p0[n], cv, p0[s]);
    const float hxx = d2v(p0[wv], cv, p0[e]);
    const float dz_yp = (pp[s] - pm[s]) / 2.f;
    const float dz_ym = (pp[n] - pm[n]) / 2.f;
    const float hyz = (dz_yp - dz_ym) / 2.f;
    const float dz_xp = (pp[e] - pm[e]) / 2.f;
    const float dz_xm = (pp[wv] - pm[wv]) / 2.f;
    const float hxz = (dz_xp - dz_xm) / 2.f;
    const float dy_xp = (p0[s + 1] - p0[n + 1]) / 2.f;
    const float dy_xm = (p0[s - 1] - p0[n - 1]) / 2.f;
    const float hxy = (dy_xp - dy_xm) / 2.f;
    h[0] = hzz * w[0];
    h[1] = hyy * w[1];
    h[2] = hxx * w[2];
    h[3] = hyz * w[3];
    h[4] = hxz * w[4];
    h[5] = hxy * w[5];
}

// Boundary flags of a voxel: d1_cen_adj negates the edge-replicated value one
// step outside the volume (G(-1) = -g[0], G(n) = -g[n-1]).
struct Edge {
    float zlo, zhi, ylo, yhi, xlo, xhi;  // -1 at the matching volume edge, else +1
};

// d1_cen_adj along a of (inner) then b of a staged component; a/b steps are
// in-tile offsets (da, db are the index steps of axes a and b; planes for b = z).
__device__ __forceinline__ float inner_s(const float* p, int c, int da, float slo, float shi, float w) {
    return __fsub_rn(slo * wmul(p[c - da], w), shi * wmul(p[c + da], w)) / 2.f;
}

// Hessian3D.adjoint at tile-local (ly, lx) from staged components:
// g0/g3/g4 as (prev, cur, next) plane triples, g1/g2/g5 in plane z.
__device__ __forceinline__ float hess_adj_smem(const float* g0m, const float* g0c, const float* g0p,
                                               const float* g1, const float* g2,
                                               const float* g3m, const float* g3p,
                                               const float* g4m, const float* g4p, const float* g5,
                                               int ly, int lx, const Edge& e, const float w[6]) {
    const int c = ly * kHX + lx;
    const float azz = d2v(wmul(g0m[c], w[0]), wmul(g0c[c], w[0]), wmul(g0p[c], w[0]));
    const float ayy = d2v(wmul(g1[c - kHX], w[1]), wmul(g1[c], w[1]), wmul(g1[c + kHX], w[1]));
    const float axx = d2v(wmul(g2[c - 1], w[2]), wmul(g2[c], w[2]), wmul(g2[c + 1], w[2]));
    // yz: outer z (planes; at a z edge the staged neighbour plane is plane z
    // itself and the row is negated), inner y
    const float ayz = __fsub_rn(e.zlo * inner_s(g3m, c, kHX, e.ylo, e.yhi, w[3]),
                                e.zhi * inner_s(g3p, c, kHX, e.ylo, e.yhi, w[3])) / 2.f;
    // xz: outer z, inner x
    const float axz = __fsub_rn(e.zlo * inner_s(g4m, c, 1, e.xlo, e.xhi, w[4]),
                                e.zhi * inner_s(g4p, c, 1, e.xlo, e.xhi, w[4])) / 2.f;
    // xy: outer y (rows c -+ kHX in plane z), inner x
    const float axy = __fsub_rn(e.ylo * inner_s(g5, c - kHX, 1, e.xlo, e.xhi, w[5]),
                                e.yhi * inner_s(g5, c + kHX, 1, e.xlo, e.xhi, w[5])) / 2.f;
    return __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(azz, ayy), axx), ayz), axz), axy);
}

// ---- software pipeline ------------------------------------------------------

__device__ __forceinline__ void cpa4(float* dst, const float* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpa_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int N>
struct Ptrs {
    const float* p[N > 0 ? N : 1];
};

// Position in this CTA's stream of (tile, stage).  Stage s of a tile with
// planes [z0, z1) carries halo plane clamp(z0 - 1 + s) and, for s >= 2, the
// centre operands of plane z0 + s - 2, which is computed when stage s is
// consumed; a tile has (z1 - z0) + 2 stages.  The in-plane offsets of this
// thread's halo slots and centre voxel are set once per tile.
struct StageCursor {
    int64_t tile, x0, y0, z0, z1;
    int s, S;
    int hoff[2];  // in-plane offsets of the thread's halo slots (clamped; a plane has < 2^31 voxels)
    int coff;     // in-plane offset of the thread's voxel, -1 outside the volume
    __device__ __forceinline__ void set(int64_t t, const TileGeo& g, const Dims& d, const int ly[2],
                                        const int lx[2], int tx, int ty) {
        tile = t;
        s = 0;
        if (t < g.ntiles) {
            const int64_t bx = t % g.ntx, r = t / g.ntx, by = r % g.nty, bz = r / g.nty;
            x0 = bx * kTX;
            y0 = by * kTY;
            z0 = bz * kZChunk;
            z1 = min(z0 + kZChunk, d.nz);
            S = (int)(z1 - z0) + 2;
#pragma unroll
            for (int u = 0; u < 2; ++u)
                hoff[u] = (int)(clampi(y0 - 1 + ly[u], d.ny) * d.nx + clampi(x0 - 1 + lx[u], d.nx));
            const int64_t x = x0 + tx, y = y0 + ty;
            coff = (x < d.nx && y < d.ny) ? (int)(y * d.nx + x) : -1;
        }
    }
};

// Dynamic shared memory of one pipeline: NH halo fields x D planes, NC
// centre operands x D planes, NW working fields x 4 planes (NW = 0: the
// staged planes are used in place).
template <int NH, int NW, int NC, int D>
struct PipeLayout {
    static constexpr int kH = NH * D * kPL;
    static constexpr int kC = NC * D * kTX * kTY;
    static constexpr int kW = NW * 4 * kPL;
    static constexpr size_t bytes = (size_t)(kH + kC + kW) * sizeof(float);
};

// Runs the stream.  body(z, x, y, i, cv[NC], W) computes plane z at (x, y)
// (linear index i) with W[3 f + k] = field f at plane z - 1 + k
// (shared-memory planes of kHX x kHY).  All threads run every stage (one
// barrier each).
//
// NW > 0: conv(raw[NH], out[NW]) turns the thread's own staged halo values
// into NW working fields in a 4-plane ring; a staged slot is consumed by the
// thread that copied it, so it is refilled at once: stages run D ahead.
// NW == 0: the body reads the staged planes directly (NH fields).  A slot is
// free only after every thread has finished the body that read it, i.e.
// after the next barrier: stage g - 3 + D is issued at step g >= 3 into the
// slot of stage g - 3, so stages run D - 3 ahead.
template <int NH, int NW, int NC, int D, class CONV, class BODY>
__device__ __forceinline__ void hess_pipeline(const Dims& d, const Ptrs<NH>& hs, const Ptrs<NC>& cs,
                                              CONV conv, BODY body) {
    constexpr bool kDirect = NW == 0;
    constexpr int NF = kDirect ? NH : NW;  // fields the body sees
    static_assert(kDirect ? D >= 4 : D >= 2, "pipeline depth");
    extern __shared__ float smf[];
    float* hraw = smf;
    float* craw = hraw + PipeLayout<NH, NW, NC, D>::kH;
    float* work = craw + PipeLayout<NH, NW, NC, D>::kC;
    const TileGeo g(d);
    const int tid = threadIdx.x, tx = tid % kTX, ty = tid / kTX;
    const int64_t plane = d.ny * d.nx;
    int q[2], ly[2], lx[2];
    bool okq[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
        q[u] = tid + u * kTX * kTY;
        okq[u] = q[u] < kPL;
        ly[u] = q[u] / kHX;
        lx[u] = q[u] - ly[u] * kHX;
    }
    StageCursor is, cc;
    is.set(blockIdx.x, g, d, ly, lx, tx, ty);
    cc = is;
    int gi = 0, gc = 0;
    auto issue = [&]() {
        if (is.tile < g.ntiles) {
            const int slot = gi % D;
            const int64_t zh = clampi(is.z0 - 1 + is.s, d.nz) * plane;
#pragma unroll
            for (int a = 0; a < NH; ++a) {
                const float* base = hs.p[a] + zh;
                float* dst = hraw + (a * D + slot) * kPL;
#pragma unroll
                for (int u = 0; u < 2; ++u)
                    if (okq[u]) cpa4(dst + q[u], base + is.hoff[u]);
            }
            if (NC > 0 && is.s >= 2 && is.coff >= 0) {
                const int64_t zc = (is.z0 + is.s - 2) * plane;
#pragma unroll
                for (int c = 0; c < NC; ++c) cpa4(&craw[(c * D + slot) * (kTX * kTY) + tid], cs.p[c] + zc + is.coff);
            }
            if (++is.s == is.S) is.set(is.tile + gridDim.x, g, d, ly, lx, tx, ty);
            ++gi;
        }
        cpa_commit();
    };
#pragma unroll 1
    for (int k = 0; k < D; ++k) issue();
#pragma unroll 1
    while (cc.tile < g.ntiles) {
        const int slot = gc % D;
        if constexpr (kDirect) {
            cpa_wait<D - 4>();
        } else {
            cpa_wait<D - 1>();
            const int ws = gc & 3;
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                if (!okq[u]) continue;
                float raw[NH], out[NW > 0 ? NW : 1];
#pragma unroll
                for (int a = 0; a < NH; ++a) raw[a] = hraw[(a * D + slot) * kPL + q[u]];
                conv(raw, out);
#pragma unroll
                for (int f = 0; f < NW; ++f) work[(f * 4 + ws) * kPL + q[u]] = out[f];
            }
        }
        __syncthreads();
        if constexpr (kDirect) {
            if (gc >= 3) issue();  // into the slot of stage gc - 3, read last at step gc - 1
            else cpa_commit();
        }
        if (cc.s >= 2 && cc.coff >= 0) {
            const int64_t z = cc.z0 + cc.s - 2;
            const int64_t x = cc.x0 + tx, y = cc.y0 + ty;
            float cv[NC > 0 ? NC : 1];
#pragma unroll
            for (int c = 0; c < NC; ++c) cv[c] = craw[(c * D + slot) * (kTX * kTY) + tid];
            const float* W[3 * NF];
#pragma unroll
            for (int f = 0; f < NF; ++f)
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    if constexpr (kDirect) W[3 * f + k] = hraw + (f * D + (gc - 2 + k) % D) * kPL;
                    else W[3 * f + k] = work + (f * 4 + ((gc - 2 + k) & 3)) * kPL;
                }
            body(z, x, y, z * plane + cc.coff, cv, W);
        }
        if (++cc.s == cc.S) cc.set(cc.tile + gridDim.x, g, d, ly, lx, tx, ty);
        ++gc;
        if constexpr (!kDirect) issue();
    }
    cpa_wait<0>();
}

constexpr int kDualDepth = 4, kLossDepth = 8;
using DualLayout = PipeLayout<2, 1, 6, kDualDepth>;
using LossLayout = PipeLayout<1, 1, 0, kLossDepth>;

// y2 = proj(y2 + sigma H x_bar), x_bar = x + theta (x - x_prev) formed at staging.
template <int NORM>
__global__ void __launch_bounds__(256) k_hess_dual_p(PdhgDev* s, float* y2,
                                                     const float* __restrict__ xc,
                                                     const float* __restrict__ xp, Dims d, W6 w,
                                                     float alpha) {
    if (s->stop) return;
    const float sg = (float)s->sigma, th = (float)s->theta;
    const int64_t n = d.nz * d.ny * d.nx;
    Ptrs<2> hs{{xc, xp}};
    Ptrs<6> cs;
#pragma unroll
    for (int c = 0; c < 6; ++c) cs.p[c] = y2 + c * n;
    const int tx = threadIdx.x % kTX, ty = threadIdx.x / kTX;
    hess_pipeline<2, 1, 6, kDualDepth>(
        d, hs, cs, [&](const float* r, float* o) { o[0] = xbar_of(r[0], r[1], th); },
        [&](int64_t, int64_t, int64_t, int64_t i, const float* cv, const float* const* W) {
            float h[6];
            hess6_smem(W[0], W[1], W[2], ty + 1, tx + 1, w.w, h);
            if constexpr (NORM == 0) {
#pragma unroll
                for (int c = 0; c < 6; ++c) y2[c * n + i] = fminf(fmaxf(dual_arg(cv[c], sg, h[c]), -alpha), alpha);
            } else {
                float v[6];
                float ss = 0.f;
#pragma unroll
                for (int c = 0; c < 6; ++c) {
                    v[c] = dual_arg(cv[c], sg, h[c]);
                    ss += v[c] * v[c];
                }
                const float sc = fmaxf(sqrtf(ss + 1e-12f) / alpha, 1.f);
#pragma unroll
                for (int c = 0; c < 6; ++c) y2[c * n + i] = v[c] / sc;
            }
        });
}

// Per-CTA FP64 partial sum into slot `slot`; with a grid smaller than
// kPdhgGrid, CTA 0 zeroes the slots no CTA writes (the fold sums all).
__device__ __forceinline__ void put_slot(PdhgDev* s, int slot, double v) {
    const double b = block_sum(v);
    if (threadIdx.x == 0) s->partials[slot * kPdhgGrid + blockIdx.x] = b;
    if (blockIdx.x == 0)
        for (int i = gridDim.x + threadIdx.x; i < kPdhgGrid; i += blockDim.x) s->partials[slot * kPdhgGrid + i] = 0.0;
}

// ||A x_new - A x||^2 and ||H (x_new - x)||^2 (z axis walked in registers).
template <class IDX>
__global__ void __launch_bounds__(256) k_hess_dk_r(PdhgDev* s, const float* __restrict__ axn,
                                                   const float* __restrict__ axc, int64_t m,
                                                   const float* __restrict__ xn,
                                                   const float* __restrict__ xc, Dims d, W6 w,
                                                   int slot_a, int slot_l) {
    if (s->stop) return;
    double a2 = 0.0, l2 = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double dd = (double)axn[i] - (double)axc[i];
        a2 += dd * dd;
    }
    hess_zwalk<IDX, 1>(
        d, w, [&](IDX i) { return make_float2(__ldg(xn + i), __ldg(xc + i)); },
        [](const float2& r, int) { return r.x - r.y; },
        [&](IDX, const float (*h)[6]) {
            // the six squares of one voxel in FP32, the sum over voxels in FP64
            float v = 0.f;
#pragma unroll
            for (int k = 0; k < 6; ++k) v = fmaf(h[0][k], h[0][k], v);
            l2 += (double)v;
        });
    put_slot(s, slot_a, a2);
    put_slot(s, slot_l, l2);
}

template <int NORM>
__global__ void __launch_bounds__(256) k_hess_regloss_p(PdhgDev* s, const float* __restrict__ x,
                                                        Dims d, W6 w, int kk, int slot) {
    if (!(kk < s->final_iter && !(s->converged && kk == s->final_iter - 1))) return;
    double acc = 0.0;
    Ptrs<1> hs{{x}};
    Ptrs<0> cs{{nullptr}};
    const int tx = threadIdx.x % kTX, ty = threadIdx.x / kTX;
    hess_pipeline<1, 1, 0, kLossDepth>(
        d, hs, cs, [&](const float* r, float* o) { o[0] = r[0]; },
        [&](int64_t, int64_t, int64_t, int64_t, const float*, const float* const* W) {
            float h[6];
            hess6_smem(W[0], W[1], W[2], ty + 1, tx + 1, w.w, h);
            if constexpr (NORM == 0) {
                float v = 0.f;
#pragma unroll
                for (int c = 0; c < 6; ++c) v += fabsf(h[c]);
                acc += (double)v;
            } else {
                float ss = 0.f;
#pragma unroll
                for (int c = 0; c < 6; ++c) ss += h[c] * h[c];
                acc += (double)sqrtf(ss + 1e-12f);
            }
        });
    put_slot(s, slot, acc);
}

// H^T y2 over this CTA's tiles from staged planes: components 0, 3, 4 (read
// at z -+ 1) in rings of three planes, components 1, 2, 5 (read in plane z
// only) one plane each, a one-plane register prefetch.  body(i, lt, cv)
// receives the adjoint at interior voxel i (the float operations of
// hess_adj_gen) and the NC centre operands cen[c][i], which are prefetched
// into registers one plane ahead with the y2 halo values (a load issued in
// the body would wait a full memory latency per plane).
//
// The walk is bound by instruction issue, so its index arithmetic is kept
// lean: IDX is the type of element offsets (uint32_t when 6 n < 2^32, which
// the launchers check, else int64_t), every per-tile quantity is set once
// per tile, plane offsets advance by additions and the three ring slots
// rotate instead of being recomputed modulo 3.
template <class IDX, int NC, class Body>
__device__ __forceinline__ void hess_adj_walk_c(const float* __restrict__ y2, const Dims& d, const W6& w,
                                                const float* const* cen, const Body& body) {
    __shared__ float rz[3][3][kPL];  // components 0, 3, 4
    __shared__ float pz[3][kPL];     // components 1, 2, 5
    const IDX n = (IDX)(d.nz * d.ny * d.nx), plane = (IDX)(d.ny * d.nx);
    const int nz = (int)d.nz;
    const TileGeo g(d);
    const int tid = threadIdx.x, tx = tid % kTX, ty = tid / kTX;
    // this thread's two halo-window slots (the second exists for tid < kPL - 256)
    const int q1 = tid + 256;
    const bool ok1 = q1 < kPL;
    const int ly0 = tid / kHX, lx0 = tid - ly0 * kHX, ly1 = q1 / kHX, lx1 = q1 - ly1 * kHX;
    const float* const y2c1 = y2 + n;
    const float* const y2c2 = y2 + 2 * n;
    const float* const y2c3 = y2 + 3 * n;
    const float* const y2c4 = y2 + 4 * n;
    const float* const y2c5 = y2 + 5 * n;
    for (int64_t tile = blockIdx.x; tile < g.ntiles; tile += gridDim.x) {
        const int64_t bx = tile % g.ntx, r = tile / g.ntx, by = r % g.nty, bz = r / g.nty;
        const int64_t x0 = bx * kTX, y0 = by * kTY;
        const int z0 = (int)(bz * kZChunk);
        const int z1 = z0 + kZChunk < nz ? z0 + kZChunk : nz;
        const int64_t x = x0 + tx, y = y0 + ty;
        const bool in = x < d.nx && y < d.ny;
        const IDX ipl = in ? (IDX)(y * d.nx + x) : (IDX)0;
        Edge e;
        e.ylo = y == 0 ? -1.f : 1.f;
        e.yhi = y == d.ny - 1 ? -1.f : 1.f;
        e.xlo = x == 0 ? -1.f : 1.f;
        e.xhi = x == d.nx - 1 ? -1.f : 1.f;
        const IDX off0 = (IDX)(clampi(y0 - 1 + ly0, d.ny) * d.nx + clampi(x0 - 1 + lx0, d.nx));
        const IDX off1 = ok1 ? (IDX)(clampi(y0 - 1 + ly1, d.ny) * d.nx + clampi(x0 - 1 + lx1, d.nx)) : (IDX)0;
        // the two slots' values of one component base at plane offset zo
        auto ld = [&](const float* cb, IDX zo, float v[2]) {
            v[0] = __ldg(cb + (zo + off0));
            v[1] = ok1 ? __ldg(cb + (zo + off1)) : 0.f;
        };
        auto st = [&](float* pl, const float v[2]) {
            pl[tid] = v[0];
            if (ok1) pl[q1] = v[1];
        };
        float p0[2], p3[2], p4[2], p1[2], p2[2], p5[2];
        {
            const IDX zb = (IDX)(z0 > 0 ? z0 - 1 : 0) * plane;
            ld(y2, zb, p0);
            ld(y2c3, zb, p3);
            ld(y2c4, zb, p4);
            st(rz[0][0], p0);
            st(rz[1][0], p3);
            st(rz[2][0], p4);
            const IDX zc = (IDX)z0 * plane;
            ld(y2, zc, p0);
            ld(y2c3, zc, p3);
            ld(y2c4, zc, p4);
            st(rz[0][1], p0);
            st(rz[1][1], p3);
            st(rz[2][1], p4);
        }
        float cv[NC > 0 ? NC : 1], cn[NC > 0 ? NC : 1];
        IDX zo = (IDX)z0 * plane;  // offset of plane z
        {
            const IDX zn = (IDX)(z0 + 1 < nz ? z0 + 1 : nz - 1) * plane;
            ld(y2, zn, p0);
            ld(y2c3, zn, p3);
            ld(y2c4, zn, p4);
            ld(y2c1, zo, p1);
            ld(y2c2, zo, p2);
            ld(y2c5, zo, p5);
#pragma unroll
            for (int c = 0; c < NC; ++c) cn[c] = in ? __ldg(cen[c] + (zo + ipl)) : 0.f;
        }
        int sp = 0, sc = 1, sn = 2;  // ring slots of planes z - 1, z, z + 1
        for (int z = z0; z < z1; ++z) {
#pragma unroll
            for (int c = 0; c < NC; ++c) cv[c] = cn[c];
            st(rz[0][sn], p0);
            st(rz[1][sn], p3);
            st(rz[2][sn], p4);
            st(pz[0], p1);
            st(pz[1], p2);
            st(pz[2], p5);
            __syncthreads();
            const IDX zi = zo;  // plane z
            zo += plane;        // plane z + 1
            if (z + 1 < z1) {
                const IDX zn = z + 2 < nz ? zo + plane : zo;  // clamp(z + 2)
                ld(y2, zn, p0);
                ld(y2c3, zn, p3);
                ld(y2c4, zn, p4);
                ld(y2c1, zo, p1);
                ld(y2c2, zo, p2);
                ld(y2c5, zo, p5);
#pragma unroll
                for (int c = 0; c < NC; ++c) cn[c] = in ? __ldg(cen[c] + (zo + ipl)) : 0.f;
            }
            if (in) {
                e.zlo = z == 0 ? -1.f : 1.f;
                e.zhi = z == nz - 1 ? -1.f : 1.f;
                const float lt = hess_adj_smem(rz[0][sp], rz[0][sc], rz[0][sn], pz[0], pz[1],
                                               rz[1][sp], rz[1][sn], rz[2][sp], rz[2][sn], pz[2],
                                               ty + 1, tx + 1, e, w.w);
                body(zi + ipl, lt, cv);
            }
            __syncthreads();
            const int t = sp;
            sp = sc;
            sc = sn;
            sn = t;
        }
    }
}

template <class IDX, class Body>
__device__ __forceinline__ void hess_adj_walk(const float* __restrict__ y2, const Dims& d, const W6& w,
                                              const Body& body) {
    hess_adj_walk_c<IDX, 0>(y2, d, w, nullptr, [&](IDX i, float lt, const float*) { body(i, lt); });
}

// x_new = max(0, x - tau (A^T y1 + H^T y2)) and its FP64 sums.
template <class IDX>
__global__ void __launch_bounds__(256) k_hess_primal_t(PdhgDev* s, const float* __restrict__ xc,
                                                       const float* __restrict__ aty,
                                                       const float* __restrict__ y2,
                                                       float* __restrict__ xn, Dims d, W6 w,
                                                       int s_dx2, int s_xc2, int s_xn2) {
    if (s->stop) return;
    const float tau = (float)s->tau;
    double dx2 = 0.0, xc2 = 0.0, xn2 = 0.0;
    const float* cen[2] = {xc, aty};
    hess_adj_walk_c<IDX, 2>(y2, d, w, cen, [&](IDX i, float lt, const float* cv) {
        const float a = cv[0];
        const float gr = __fadd_rn(cv[1], lt);
        const float v = primal_of(a, tau, gr);
        xn[i] = v;
        const float dd = v - a;
        dx2 += (double)dd * dd;
        xc2 += (double)a * a;
        xn2 += (double)v * v;
    });
    put_slot(s, s_dx2, dx2);
    put_slot(s, s_xc2, xc2);
    put_slot(s, s_xn2, xn2);
}

// Hessian3D.adjoint of six stored components on the staged tile walk:
// bit-identical to the per-voxel global-memory form (hess_adj_gen).
template <class IDX>
__global__ void __launch_bounds__(256) k_hessian_adj_t(const float* __restrict__ hw, float* __restrict__ out,
                                                       Dims d, W6 w) {
    hess_adj_walk<IDX>(hw, d, w, [&](IDX i, float lt) { out[i] = lt; });
}


// ---- dual and primal update in one z-walk -----------------------------------
//
// y2_out = proj(y2_in + sigma H x_bar) and x_new = max(0, x - tau (A^T y1 +
// H^T y2_out)) for one iteration, without y2_out making a round trip through
// global memory between the two: per tile the CTA walks z, staging x_bar with
// a two-voxel halo (36 x 12), evaluating y2_out on the one-voxel halo (34 x
// 10) of each plane from it, and H^T y2_out of the tile's interior from the
// last three y2_out planes.  Halo values of y2_out are recomputed by every
// tile that needs them (at the clamped coordinate, which is the value the
// staged adjoint reads there), so y2 is double-buffered: y2_in is read, never
// written, and tiles never see a neighbour's new values.  The float
// operations are those of k_hess_dual_p and k_hess_primal_t (bit-identical
// results), and y2_out is written once, by the tile that owns each voxel.
constexpr int kH2X = kTX + 4, kH2Y = kTY + 4, kPL2 = kH2X * kH2Y;

// hess6_smem on a plane of row stride S.
template <int S>
__device__ __forceinline__ void hess6_at(const float* pm, const float* p0, const float* pp, int c,
                                         const float w[6], float h[6]) {
    const int n = c - S, s = c + S, wv = c - 1, e = c + 1;
    const float cv = p0[c];
    const float hzz = d2v(pm[c], cv, pp[c]);
    const float hyy = d2v(p0[n], cv, p0[s]);
    const float hxx = d2v(p0[wv], cv, p0[e]);
    const float dz_yp = (pp[s] - pm[s]) / 2.f;
    const float dz_ym = (pp[n] - pm[n]) / 2.f;
    const float hyz = (dz_yp - dz_ym) / 2.f;
    const float dz_xp = (pp[e] - pm[e]) / 2.f;
    const float dz_xm = (pp[wv] - pm[wv]) / 2.f;
    const float hxz = (dz_xp - dz_xm) / 2.f;
    const float dy_xp = (p0[s + 1] - p0[n + 1]) / 2.f;
    const float dy_xm = (p0[s - 1] - p0[n - 1]) / 2.f;
    const float hxy = (dy_xp - dy_xm) / 2.f;
    h[0] = hzz * w[0];
    h[1] = hyy * w[1];
    h[2] = hxx * w[2];
    h[3] = hyz * w[3];
    h[4] = hxz * w[4];
    h[5] = hxy * w[5];
}

template <int NORM>
__global__ void __launch_bounds__(256) k_hess_dual_primal(
    PdhgDev* s, const float* __restrict__ y2_in, float* __restrict__ y2_out,
    const float* __restrict__ xc, const float* __restrict__ xp, const float* __restrict__ aty,
    float* __restrict__ xn, Dims d, W6 w, float alpha, int s_dx2, int s_xc2, int s_xn2) {
    if (s->stop) return;
    __shared__ float xb[4][kPL2];     // x_bar planes, ring slot = plane & 3
    __shared__ float yn[6][4][kPL];   // y2_out planes, ring slot = plane & 3
    const float sg = (float)s->sigma, th = (float)s->theta, tau = (float)s->tau;
    const int64_t n = d.nz * d.ny * d.nx, plane = d.ny * d.nx;
    const TileGeo g(d);
    const int tid = threadIdx.x, tx = tid % kTX, ty = tid / kTX;
    double dx2 = 0.0, xc2 = 0.0, xn2 = 0.0;
    for (int64_t tile = blockIdx.x; tile < g.ntiles; tile += gridDim.x) {
        const int64_t bx = tile % g.ntx, rr = tile / g.ntx, by = rr % g.nty, bz = rr / g.nty;
        const int64_t x0 = bx * kTX, y0 = by * kTY, z0 = bz * kZChunk;
        const int64_t z1 = min(z0 + kZChunk, d.nz);
        // this thread's x_bar staging slots (two-voxel halo, clamped coordinates)
        int64_t o2[2];
        bool k2[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int q = tid + u * 256;
            k2[u] = q < kPL2;
            const int sy = q / kH2X, sx = q - sy * kH2X;
            o2[u] = clampi(y0 - 2 + sy, d.ny) * d.nx + clampi(x0 - 2 + sx, d.nx);
        }
        // this thread's y2_out positions (one-voxel halo): the clamped voxel,
        // its stencil centre in the x_bar plane, and whether it owns the voxel
        int64_t o1[2];
        int c2[2];
        bool k1[2], own[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int q = tid + u * 256;
            k1[u] = q < kPL;
            const int ly = q / kHX, lx = q - ly * kHX;
            const int64_t yy = y0 - 1 + ly, xx = x0 - 1 + lx;
            const int64_t gy = clampi(yy, d.ny), gx = clampi(xx, d.nx);
            o1[u] = gy * d.nx + gx;
            c2[u] = (int)((gy - (y0 - 2)) * kH2X + (gx - (x0 - 2)));
            own[u] = ly >= 1 && ly <= kTY && lx >= 1 && lx <= kTX && yy < d.ny && xx < d.nx;
        }
        const int64_t x = x0 + tx, y = y0 + ty;
        const bool in = x < d.nx && y < d.ny;
        const int64_t ipl = y * d.nx + x;
        Edge e;
        e.ylo = y == 0 ? -1.f : 1.f;
        e.yhi = y == d.ny - 1 ? -1.f : 1.f;
        e.xlo = x == 0 ? -1.f : 1.f;
        e.xhi = x == d.nx - 1 ? -1.f : 1.f;
        const int64_t qa = max(z0 - 1, (int64_t)0), qb = min(z1, d.nz - 1);  // y2_out planes
        const int64_t pa = max(qa - 1, (int64_t)0), pb = min(qb + 1, d.nz - 1);  // x_bar planes
        // Global operands are loaded one step ahead into the registers the
        // current step has just consumed: x and x_prev of the next x_bar plane
        // (issued right after staging), y2_in of the next dual plane (after
        // the dual update), x and A^T y1 of the next primal plane (after the
        // primal update), so every load is in flight across a barrier and a
        // plane of arithmetic.
        auto load_x = [&](int64_t p, float ra[2], float rp[2]) {
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                if (!k2[u]) continue;
                const int64_t i = p * plane + o2[u];
                ra[u] = __ldg(xc + i);
                rp[u] = __ldg(xp + i);
            }
        };
        auto load_y = [&](int64_t q, float ry[2][6]) {
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                if (!k1[u]) continue;
                const int64_t i = q * plane + o1[u];
#pragma unroll
                for (int c = 0; c < 6; ++c) ry[u][c] = __ldg(y2_in + c * n + i);
            }
        };
        auto load_pr = [&](int64_t z, float& a, float& at) {
            if (!in || z < z0 || z >= z1) return;
            const int64_t i = z * plane + ipl;
            a = __ldg(xc + i);
            at = __ldg(aty + i);
        };
        auto dual_plane = [&](int64_t q, const float ry[2][6]) {
            const int64_t qm = clampi(q - 1, d.nz), qp = clampi(q + 1, d.nz);
            const float* pm = xb[qm & 3];
            const float* p0 = xb[q & 3];
            const float* pp = xb[qp & 3];
            const bool owned_plane = q >= z0 && q < z1;
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                if (!k1[u]) continue;
                float h[6];
                hess6_at<kH2X>(pm, p0, pp, c2[u], w.w, h);
                const int64_t i = q * plane + o1[u];
                float v[6];
                if constexpr (NORM == 0) {
#pragma unroll
                    for (int c = 0; c < 6; ++c) v[c] = fminf(fmaxf(dual_arg(ry[u][c], sg, h[c]), -alpha), alpha);
                } else {
                    float ss = 0.f;
#pragma unroll
                    for (int c = 0; c < 6; ++c) {
                        v[c] = dual_arg(ry[u][c], sg, h[c]);
                        ss += v[c] * v[c];
                    }
                    const float sc = fmaxf(sqrtf(ss + 1e-12f) / alpha, 1.f);
#pragma unroll
                    for (int c = 0; c < 6; ++c) v[c] = v[c] / sc;
                }
                const int q1 = tid + u * 256;
#pragma unroll
                for (int c = 0; c < 6; ++c) yn[c][q & 3][q1] = v[c];
                if (own[u] && owned_plane) {
#pragma unroll
                    for (int c = 0; c < 6; ++c) y2_out[c * n + i] = v[c];
                }
            }
        };
        auto primal_plane = [&](int64_t z, float a, float at) {
            if (!in || z < z0 || z >= z1) return;
            const int sm_ = (int)(clampi(z - 1, d.nz) & 3), sc_ = (int)(z & 3),
                      sp_ = (int)(clampi(z + 1, d.nz) & 3);
            e.zlo = z == 0 ? -1.f : 1.f;
            e.zhi = z == d.nz - 1 ? -1.f : 1.f;
            const float lt = hess_adj_smem(yn[0][sm_], yn[0][sc_], yn[0][sp_], yn[1][sc_], yn[2][sc_],
                                           yn[3][sm_], yn[3][sp_], yn[4][sm_], yn[4][sp_], yn[5][sc_],
                                           ty + 1, tx + 1, e, w.w);
            const int64_t i = z * plane + ipl;
            const float gr = __fadd_rn(at, lt);
            const float v = primal_of(a, tau, gr);
            xn[i] = v;
            const float dd = v - a;
            dx2 += (double)dd * dd;
            xc2 += (double)a * a;
            xn2 += (double)v * v;
        };
        float rxa[2] = {0.f, 0.f}, rxp[2] = {0.f, 0.f}, ry[2][6] = {}, pra = 0.f, prt = 0.f;
        load_x(pa, rxa, rxp);
        if (pa - 1 >= qa) load_y(pa - 1, ry);
        load_pr(pa - 2, pra, prt);
        for (int64_t p = pa; p <= pb; ++p) {
            // stage x_bar plane p (two-voxel halo), then fetch the next one's inputs
            float* dst = xb[p & 3];
#pragma unroll
            for (int u = 0; u < 2; ++u)
                if (k2[u]) dst[tid + u * 256] = xbar_of(rxa[u], rxp[u], th);
            if (p + 1 <= pb) load_x(p + 1, rxa, rxp);
            __syncthreads();
            // y2_out planes whose x_bar neighbourhood is complete
            const int64_t q = p - 1;
            const bool last = p == d.nz - 1 && p >= qa && p <= qb;
            if (q >= qa && q <= qb) dual_plane(q, ry);
            if (p >= qa && p <= qb) load_y(p, ry);  // the next dual plane, or this last one
            if (last) dual_plane(p, ry);
            __syncthreads();
            // x_new planes whose y2_out neighbourhood is complete
            if (q >= qa && q <= qb) {
                primal_plane(q - 1, pra, prt);
                load_pr(q, pra, prt);  // the next primal plane
            }
            if (last) {
                // the volume's last plane: planes q and p complete together
                if (q >= qa && q <= qb) primal_plane(q, pra, prt);
                load_pr(p, pra, prt);
                primal_plane(p, pra, prt);
            }
        }
        __syncthreads();  // the rings are reused by the next tile
    }
    put_slot(s, s_dx2, dx2);
    put_slot(s, s_xc2, xc2);
    put_slot(s, s_xn2, xn2);
}

}  // namespace dk
