// Fused Y / axial pass: Y FFT -> axial FFT x OTF x IFFT -> Y IFFT in one
// kernel, one thread-block cluster per kx column, on a kx-major spectrum.
//
// After the X R2C pass the spectrum S1 holds, for every kx, the (z, y) plane
// of Nz x Ny complex values, contiguous ([Hx][Nz][Ny]).  The rest of the
// convolution for one kx is a 2-D problem on the (kz, ky) plane of the canvas
// (FZ x FY, both powers of two, Nz <= FZ / 2, Ny <= FY / 2), which a cluster
// of C = 8 CTAs holds in distributed shared memory:
//
//   A  CTA c loads its z rows [c zpc, (c + 1) zpc) of the plane (one bulk
//      copy) and transforms them along y (FY points, the signal in the first
//      half: even / odd outputs from two FY/2-point FFTs of x and x W_FY^n).
//   B  cluster barrier; CTA c gathers the columns ky in [c cpc, (c + 1) cpc)
//      of every row from the other CTAs' shared memory.
//   C  along z for each of its columns: forward FFT (half-zero split again),
//      x OTF (or conj OTF), inverse FFT, keep z < Nz.  The OTF is stored
//      kx-major ([Hx][FY][FZ]), so a column's values are contiguous.
//   D  cluster barrier; CTA c gathers its z rows of every column back.
//   E  inverse Y FFT of its rows, keep y < Ny, store in place into S1.
//
// The doubled-in-y spectrum (Nz x FY x Hx, the largest intermediate of the
// unfused passes) therefore never exists in global memory: per convolution
// the pass reads S1 and the OTF once and writes S1 once.
//
// Every FFT is warp-synchronous: a transform of L points belongs to LANES =
// L / V lanes of one warp holding V points each (V = 16 for L >= 128, else
// 8), two radix stages (V, then LANES) with one exchange through this
// transform's own shared-memory scratch, ordered by __syncwarp only.  After
// the second stage a lane holds the points its first stage of the next
// transform reads (j + LANES r), so the OTF product and the inverse follow
// in registers.  CTA-wide barriers separate the phases only.
#pragma once

#include <cooperative_groups.h>

#include "conv_impl.cuh"
#include "tma.cuh"

namespace dk {

namespace cgx = cooperative_groups;

// Default cluster: 8 CTAs of 512 threads (one CTA per SM); the alternative
// 16 CTAs of 256 threads halves each CTA's shared memory, so two CTAs (of two
// different clusters) share an SM and one's barriers overlap the other's work.
constexpr int kYZCluster = 8;
constexpr int kYZThreads = 512;

struct YZArgs {
    float2* s1t;          // [Hx][Nz][Ny], transformed in place
    const float2* otft;   // [Hx][FY][FZ]
    const float2* twy;    // W_FY^m, m < FY (global; staged in shared memory)
    const float2* twz;    // W_FZ^m, m < FZ
    int Nz, Ny, Hx;
};

// Contiguous bulk copy global -> shared (no tensor map), completion on an
// mbarrier.  Both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void fence_proxy_async_all() { asm volatile("fence.proxy.async;" ::: "memory"); }

// Bulk prefetch of a contiguous global range into L2 (16-byte aligned,
// bytes a multiple of 16).
__device__ __forceinline__ void bulk_prefetch_l2(const void* src, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

// A transform of L points by LANES lanes of one warp (see the file comment).
// v[r] holds point j + LANES r on entry and on exit; buf is the transform's
// own L-entry scratch; xs (0 or 8) separates two transforms sharing a
// half-warp in the shared-memory banks; tw is the W_{2L} table.
template <int L>
struct WarpFFT {
    static constexpr int V = L >= 128 ? 16 : 8;
    static constexpr int LANES = L / V;
    static constexpr int U = V / LANES;  // second-stage butterflies per lane
    __device__ __forceinline__ static int swz(int p, int xs) { return p ^ ((p / V) & (V - 1)) ^ xs; }

    template <int DIR>
    __device__ __forceinline__ static void run(float2 (&v)[V], float2* buf, int j, int xs,
                                               const float2* tw) {
        // stage 1 (radix V, no twiddles): butterfly j over points j + LANES r
        dft<V, DIR>(v);
        __syncwarp();  // every lane has read its inputs (they may share buf)
#pragma unroll
        for (int r = 0; r < V; ++r) buf[swz(j * V + r, xs)] = v[r];
        __syncwarp();
        // stage 2 (radix LANES): butterfly b over points b + V r, twiddle W_L^(r b)
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int b = j + LANES * u;
            float2 w[LANES];
#pragma unroll
            for (int r = 0; r < LANES; ++r) {
                const float2 x = buf[swz(b + r * V, xs)];
                if (r == 0) {
                    w[r] = x;
                } else {
                    const float2 t = tw[2 * r * b];
                    w[r] = DIR < 0 ? cmul(x, t) : cmulc(x, t);
                }
            }
            dft<LANES, DIR>(w);
            // output point b + V r = j + LANES (u + U r)
#pragma unroll
            for (int r = 0; r < LANES; ++r) v[u + U * r] = w[r];
        }
        __syncwarp();  // every lane has read the scratch
    }
};

// Shared-memory bytes of k_yz for a (FY, FZ, cluster size) instantiation.
__host__ __device__ constexpr size_t yz_smem_bytes(int FY, int FZ, int C) {
    return (size_t)(FY + FZ) * 8 + (size_t)(FZ / (2 * C)) * FY * 8 + (size_t)(FY / C) * FZ * 8;
}

// C: CTAs per cluster (launched with that cluster dimension); NT: threads.
template <int FY, int FZ, int MODE, int C, int NT>
__global__ void __launch_bounds__(NT, 512 / NT) k_yz(const __grid_constant__ YZArgs a) {
    constexpr int kYZCluster = C;
    constexpr int kYZThreads = NT;
    constexpr int kYZWarps = NT / 32;
    constexpr int LY = FY / 2, LZ = FZ / 2;
    using FY_ = WarpFFT<LY>;
    using FZ_ = WarpFFT<LZ>;
    constexpr int VY = FY_::V, NLY = FY_::LANES;
    constexpr int VZ = FZ_::V, NLZ = FZ_::LANES;
    constexpr int ZPC_MAX = FZ / (2 * kYZCluster);  // rows per CTA at Nz = FZ / 2
    constexpr int CPC = FY / kYZCluster;             // columns per CTA
    constexpr int ROWS_PER_WARP = 32 / (2 * NLY);
    constexpr int COLS_PER_WARP = 32 / (2 * NLZ);
    static_assert(CPC >= 16 && CPC <= 64, "column block");
    static_assert(NLZ == 8, "axial transforms of 8 lanes");

    extern __shared__ __align__(16) unsigned char yz_raw[];
    float2* twy = reinterpret_cast<float2*>(yz_raw);
    float2* twz = twy + FY;
    float2* A = twz + FZ;             // [ZPC_MAX][FY] rows along y
    float2* B = A + ZPC_MAX * FY;     // [CPC][FZ] columns along z (input rows first)
    __shared__ uint64_t bar;

    cgx::cluster_group cluster = cgx::this_cluster();
    const int c = (int)cluster.block_rank();
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int Nz = a.Nz, Ny = a.Ny;
    const int zpc = (Nz + kYZCluster - 1) / kYZCluster;
    const int z0 = c * zpc;
    const int nzc = max(0, min(zpc, Nz - z0));
    const int ky0 = c * CPC;
    const int64_t plane = (int64_t)Nz * Ny;
    const int ncl = gridDim.x / kYZCluster;
    const int g = blockIdx.x / kYZCluster;

    for (int i = tid; i < FY; i += blockDim.x) twy[i] = a.twy[i];
    for (int i = tid; i < FZ; i += blockDim.x) twz[i] = a.twz[i];
    if (tid == 0) {
        mbar_init(&bar, 1);
        fence_proxy_async_smem();
    }
    __syncthreads();
    auto issue_input = [&](int kx) {
        const uint32_t bytes = (uint32_t)nzc * (uint32_t)Ny * 8u;
        mbar_expect_tx(&bar, bytes);
        if (bytes) bulk_load(B, a.s1t + (int64_t)kx * plane + (int64_t)z0 * Ny, bytes, &bar);
    };
    if (tid == 0 && g < a.Hx) issue_input(g);

    bool ok = true;
    int it = 0;
    for (int kx = g; kx < a.Hx; kx += ncl, ++it) {
        // this CTA's OTF columns (contiguous, CPC x FZ values) into L2 while
        // the Y transform and the gather run; phase C reads them from there
        if (tid == 0) {
            const float2* o = a.otft + ((int64_t)kx * FY + ky0) * FZ;
            constexpr uint32_t kBytes = (uint32_t)CPC * FZ * 8u, kChunk = 32768u;
            for (uint32_t off = 0; off < kBytes; off += kChunk)
                bulk_prefetch_l2(reinterpret_cast<const char*>(o) + off, kBytes - off < kChunk ? kBytes - off : kChunk);
        }
        // ---- A: forward Y transform of this CTA's rows: B (input) -> A ----
        ok = mbar_wait_bounded(&bar, (uint32_t)(it & 1)) && ok;
        {
            const int sub = lane % (2 * NLY), h = sub / NLY, j = sub % NLY;
            const int xs = NLY == 8 ? 8 * h : 0;
            for (int r0 = warp * ROWS_PER_WARP; r0 < zpc; r0 += kYZWarps * ROWS_PER_WARP) {
                const int row = r0 + lane / (2 * NLY);
                const bool act = row < nzc;
                float2 v[VY];
#pragma unroll
                for (int r = 0; r < VY; ++r) {
                    const int n = j + NLY * r;
                    float2 x = make_float2(0.f, 0.f);
                    if (act && n < Ny) {
                        x = B[row * Ny + n];
                        if (h) x = cmul(x, twy[n]);
                    }
                    v[r] = x;
                }
                // lanes past this CTA's rows take part in the warp's
                // transforms on zeros, in the scratch of row ZPC_MAX - 1,
                // which no active row of this CTA uses (row >= nzc there)
                float2* rowp = A + (act ? row : ZPC_MAX - 1) * FY;
                FY_::template run<-1>(v, rowp + h * LY, j, xs, twy);
                if (act) {
#pragma unroll
                    for (int r = 0; r < VY; ++r) rowp[2 * (j + NLY * r) + h] = v[r];
                }
                __syncwarp();
            }
        }
        fence_proxy_async_all();
        cluster.sync();

        // ---- B: gather this CTA's columns of every row: peers' A -> B ----
        {
            // eight remote loads in flight per thread, then the local stores
            const int total = Nz * CPC;
            for (int q0 = tid; q0 < total; q0 += 8 * kYZThreads) {
                float2 t[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int q = q0 + u * kYZThreads;
                    if (q < total) {
                        const int e = q % CPC, z = q / CPC;
                        const int p = z / zpc, r = z - p * zpc;
                        t[u] = cluster.map_shared_rank(A, p)[r * FY + ky0 + e];
                    }
                }
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int q = q0 + u * kYZThreads;
                    if (q < total) {
                        const int e = q % CPC, z = q / CPC;
                        B[e * FZ + (z ^ (e & 15))] = t[u];
                    }
                }
            }
        }
        __syncthreads();

        // ---- C: axial transforms of this CTA's columns ----
        {
            const int sub = lane & 15, h = sub >> 3, j = sub & 7;
            const int xs = 8 * h;
            constexpr int ROUNDS = CPC / (kYZWarps * COLS_PER_WARP);
            static_assert(ROUNDS >= 1 && CPC % (kYZWarps * COLS_PER_WARP) == 0, "rounds");
#pragma unroll 1
            for (int rd = 0; rd < ROUNDS; ++rd) {
                const int col = (rd * kYZWarps + warp) * COLS_PER_WARP + (lane >> 4);
                float2* cb = B + col * FZ;
                float2 v[VZ];
#pragma unroll
                for (int r = 0; r < VZ; ++r) {
                    const int n = j + NLZ * r;
                    float2 x = make_float2(0.f, 0.f);
                    if (n < Nz) {
                        x = cb[n ^ (col & 15)];
                        if (h) x = cmul(x, twz[n]);
                    }
                    v[r] = x;
                }
                FZ_::template run<-1>(v, cb + h * LZ, j, xs, twz);
                {
                    // OTF at this lane's points kz = 2 m + h, m = j + 8 r (L2)
                    const float2* op = a.otft + ((int64_t)kx * FY + ky0 + col) * FZ + h;
                    float2 o[VZ];
#pragma unroll
                    for (int r = 0; r < VZ; ++r) o[r] = __ldg(op + 2 * (j + NLZ * r));
#pragma unroll
                    for (int r = 0; r < VZ; ++r) v[r] = MODE == COL_OTF ? cmul(v[r], o[r]) : cmulc(v[r], o[r]);
                }
                FZ_::template run<+1>(v, cb + h * LZ, j, xs, twz);
                // y[n] = a0[n] + W_FZ^-n a1[n]: lane h keeps r in [h VZ/2, (h+1) VZ/2)
                float2 y[VZ / 2];
#pragma unroll
                for (int i = 0; i < VZ / 2; ++i) {
                    // static register indices: select rather than index by h
                    const float2 lo = v[i], hi = v[VZ / 2 + i];
                    const float2 send = h ? lo : hi;
                    float2 got;
                    got.x = __shfl_xor_sync(0xffffffffu, send.x, NLZ);
                    got.y = __shfl_xor_sync(0xffffffffu, send.y, NLZ);
                    const float2 mine = h ? hi : lo;
                    const float2 a0 = h ? got : mine, a1 = h ? mine : got;
                    const int n = j + NLZ * (h * (VZ / 2) + i);
                    y[i] = cadd(a0, cmulc(a1, twz[n]));
                }
                __syncthreads();  // every warp is done with its scratch of this round
                // kept z rows, [z][col ^ (z & 15)] in the first Nz * CPC entries of B
#pragma unroll
                for (int i = 0; i < VZ / 2; ++i) {
                    const int n = j + NLZ * (h * (VZ / 2) + i);
                    if (n < Nz) B[n * CPC + (col ^ (n & 15))] = y[i];
                }
            }
        }
        cluster.sync();

        // ---- D: gather this CTA's rows of every column: peers' B -> A ----
        {
            const int total = nzc * FY;
            for (int q0 = tid; q0 < total; q0 += 8 * kYZThreads) {
                float2 t[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int q = q0 + u * kYZThreads;
                    if (q < total) {
                        const int e = q % CPC, p = (q / CPC) % kYZCluster, r = q / FY;
                        const int z = z0 + r;
                        t[u] = cluster.map_shared_rank(B, p)[z * CPC + (e ^ (z & 15))];
                    }
                }
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int q = q0 + u * kYZThreads;
                    if (q < total) A[q] = t[u];  // q = r FY + p CPC + e
                }
            }
        }
        fence_proxy_async_all();
        cluster.sync();
        // every CTA has read this CTA's B: stream the next column's rows in
        if (tid == 0 && kx + ncl < a.Hx) issue_input(kx + ncl);

        // ---- E: inverse Y transform of this CTA's rows, store y < Ny ----
        {
            const int sub = lane % (2 * NLY), h = sub / NLY, j = sub % NLY;
            const int xs = NLY == 8 ? 8 * h : 0;
            for (int r0 = warp * ROWS_PER_WARP; r0 < zpc; r0 += kYZWarps * ROWS_PER_WARP) {
                const int row = r0 + lane / (2 * NLY);
                const bool act = row < nzc;
                float2* rowp = A + (act ? row : ZPC_MAX - 1) * FY;
                float2 v[VY];
#pragma unroll
                for (int r = 0; r < VY; ++r) v[r] = act ? rowp[2 * (j + NLY * r) + h] : make_float2(0.f, 0.f);
                FY_::template run<+1>(v, rowp + h * LY, j, xs, twy);
                float2* dst = a.s1t + (int64_t)kx * plane + (int64_t)(z0 + row) * Ny;
#pragma unroll
                for (int i = 0; i < VY / 2; ++i) {
                    const float2 lo = v[i], hi = v[VY / 2 + i];
                    const float2 send = h ? lo : hi;
                    float2 got;
                    got.x = __shfl_xor_sync(0xffffffffu, send.x, NLY);
                    got.y = __shfl_xor_sync(0xffffffffu, send.y, NLY);
                    const float2 mine = h ? hi : lo;
                    const float2 a0 = h ? got : mine, a1 = h ? mine : got;
                    const int n = j + NLY * (h * (VY / 2) + i);
                    if (act && ok && n < Ny) dst[n] = cadd(a0, cmulc(a1, twy[n]));
                }
                __syncwarp();
            }
        }
        __syncthreads();
    }
}

}  // namespace dk
