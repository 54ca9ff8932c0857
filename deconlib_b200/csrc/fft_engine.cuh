// Shared-memory Stockham FFT engine for batches of lines.
//
// A CTA holds T lines of L complex points in shared memory, element (j, t)
// (point j of line t) at phys(j, t) = j*T + (t ^ (j & (T-1))).  The XOR
// swizzle keeps both access patterns conflict-free: consecutive lines at one
// point (the butterflies and the strided-axis loads) and consecutive points
// of one line (the contiguous-axis loads).  T is a power of two.
//
// Each radix-R stage of the self-sorting (Stockham) algorithm reads point
// j + r*L/R, multiplies by the twiddle W_{Ns R}^{r (j mod Ns)}, applies a
// radix-R DFT and writes point (j div Ns) Ns R + (j mod Ns) + r Ns.  Every
// thread owns at most ceil(32/R) butterflies per stage, so it holds <= 35
// complex values in registers; a stage is read-all / barrier / write-all / barrier,
// which lets the transform run in place.  Threads per line: ceil(L / 32).
//
// Twiddles come from a table of exp(-2 pi i m / Lt) computed on the host in
// double precision (W_L^m = tw[m * tws]); no sin/cos is evaluated on the GPU.
// Radices 2, 3, 4, 5, 7, 8 and 16 are implemented.
#pragma once

#include "common.cuh"

namespace dk {

constexpr int kMaxStages = 16;

// Lengths with a compile-time radix sequence (fft_lines_static): 2^a x {1, 3,
// 5, 15} from 64 to 1024, so that a canvas rounded up to one of them grows an
// axis by at most 1/3; every other 7-smooth length takes the runtime-radix
// path.
#define DK_STATIC_LENGTHS(X) \
    X(64) X(80) X(96) X(128) X(160) X(192) X(240) X(256) X(320) X(384) X(480) X(512) X(640) X(768) \
    X(960) X(1024)
__host__ __device__ constexpr bool static_length(int L) {
#define DK_IS(n) L == n ||
    return DK_STATIC_LENGTHS(DK_IS) false;
#undef DK_IS
}
// Runtime-radix path: each thread holds ceil(kDynPPT / R) butterflies per
// stage (<= 14 values, all in registers), so a line takes ceil(L / kDynPPT)
// threads and a CTA up to kDynThreads.  (Holding 32 points per thread across
// a stage's barrier, as the compile-time path does, spilled every value to
// local memory on the runtime path and ran the strided passes at ~7 % of
// HBM bandwidth.)
constexpr int kDynPPT = 8;
constexpr int kDynThreads = 1024;

struct Axis {
    int L;                  // complex points per line
    int nst;                // radix stages
    unsigned long long rad; // radix of stage s in bits [4s, 4s+4), product == L
    int tpl;                // threads per line: ceil(L / 32), runtime path ceil(L / kDynPPT)
    int tws;                // table stride: W_L^m = tw[m * tws]
    const float2* tw;       // twiddle table (device)
    __host__ __device__ int radix(int s) const { return (int)((rad >> (4 * s)) & 15ull); }
};

__device__ __forceinline__ int phys(int j, int t, int T) { return j * T + (t ^ (j & (T - 1))); }

// Layout selector.  SW = 0: the XOR swizzle above (any power-of-two T).
// SW = 1: T = 16 lines whose rows are exactly 128 bytes, laid out as the TMA
// 128-byte swizzle writes them: 16-byte chunk (t / 2) XOR (j mod 8).  Both
// keep a warp's accesses to consecutive lines at one point conflict-free.
// SW >= 2: the XOR swizzle with a compile-time T = SW (the shifts and masks
// fold into the address arithmetic).
template <int SW>
__device__ __forceinline__ int physw(int j, int t, int T) {
    if constexpr (SW == 0) {
        return phys(j, t, T);
    } else if constexpr (SW == 1) {
        return j * 16 + ((((t >> 1) ^ (j & 7)) << 1) | (t & 1));
    } else {
        return j * SW + (t ^ (j & (SW - 1)));
    }
}

// multiply by -i (DIR < 0, forward) or +i (DIR > 0, inverse)
template <int DIR>
__device__ __forceinline__ float2 rot90(float2 a) {
    return DIR < 0 ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
}

template <int DIR>
__device__ __forceinline__ void dft2(float2& a, float2& b) {
    float2 t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

template <int DIR>
__device__ __forceinline__ void dft4(float2* v) {
    float2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    float2 t2 = cadd(v[1], v[3]), t3 = rot90<DIR>(csub(v[1], v[3]));
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
}

template <int DIR>
__device__ __forceinline__ void dft8(float2* v) {
    constexpr float h = 0.7071067811865476f;  // sqrt(1/2)
    float2 e[4] = {v[0], v[2], v[4], v[6]};
    float2 o[4] = {v[1], v[3], v[5], v[7]};
    dft4<DIR>(e);
    dft4<DIR>(o);
    // W8^1 = h (1 -+ i), W8^2 = -+ i, W8^3 = h (-1 -+ i)
    float2 o1 = DIR < 0 ? make_float2(h * (o[1].x + o[1].y), h * (o[1].y - o[1].x))
                        : make_float2(h * (o[1].x - o[1].y), h * (o[1].y + o[1].x));
    float2 o2 = rot90<DIR>(o[2]);
    float2 o3 = DIR < 0 ? make_float2(h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y))
                        : make_float2(-h * (o[3].x + o[3].y), h * (o[3].x - o[3].y));
    v[0] = cadd(e[0], o[0]);
    v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], o1);
    v[5] = csub(e[1], o1);
    v[2] = cadd(e[2], o2);
    v[6] = csub(e[2], o2);
    v[3] = cadd(e[3], o3);
    v[7] = csub(e[3], o3);
}

template <int DIR>
__device__ __forceinline__ void dft3(float2* v) {
    constexpr float s3 = 0.8660254037844386f;  // sin(2 pi / 3)
    float2 s = cadd(v[1], v[2]);
    float2 d = csub(v[1], v[2]);
    float2 m = make_float2(v[0].x - 0.5f * s.x, v[0].y - 0.5f * s.y);
    float2 r = rot90<DIR>(cscale(d, s3));
    v[0] = cadd(v[0], s);
    v[1] = cadd(m, r);
    v[2] = csub(m, r);
}

template <int DIR>
__device__ __forceinline__ void dft5(float2* v) {
    constexpr float c1 = 0.30901699437494745f, c2 = -0.8090169943749473f;
    constexpr float s1 = 0.9510565162951535f, s2 = 0.5877852522924732f;
    float2 b1 = cadd(v[1], v[4]), b2 = cadd(v[2], v[3]);
    float2 d1 = csub(v[1], v[4]), d2 = csub(v[2], v[3]);
    float2 t1 = make_float2(v[0].x + c1 * b1.x + c2 * b2.x, v[0].y + c1 * b1.y + c2 * b2.y);
    float2 t2 = make_float2(v[0].x + c2 * b1.x + c1 * b2.x, v[0].y + c2 * b1.y + c1 * b2.y);
    float2 u1 = rot90<DIR>(make_float2(s1 * d1.x + s2 * d2.x, s1 * d1.y + s2 * d2.y));
    float2 u2 = rot90<DIR>(make_float2(s2 * d1.x - s1 * d2.x, s2 * d1.y - s1 * d2.y));
    v[0] = cadd(v[0], cadd(b1, b2));
    v[1] = cadd(t1, u1);
    v[4] = csub(t1, u1);
    v[2] = cadd(t2, u2);
    v[3] = csub(t2, u2);
}

template <int DIR>
__device__ __forceinline__ void dft7(float2* v) {
    // cos / sin (2 pi j / 7), j = 1..3
    constexpr float C1 = 0.6234898018587336f, C2 = -0.22252093395631434f, C3 = -0.900968867902419f;
    constexpr float S1 = 0.7818314824680298f, S2 = 0.9749279121818236f, S3 = 0.43388373911755823f;
    float2 b1 = cadd(v[1], v[6]), b2 = cadd(v[2], v[5]), b3 = cadd(v[3], v[4]);
    float2 d1 = csub(v[1], v[6]), d2 = csub(v[2], v[5]), d3 = csub(v[3], v[4]);
    const float2 a0 = v[0];
    // m = 1: cos(1,2,3) sin(1,2,3); m = 2: cos(2,4,6)=(C2,C3,C1) sin(2,4,6)=(S2,-S3,-S1)
    // m = 3: cos(3,6,9)=(C3,C1,C2) sin(3,6,9)=(S3,-S1,S2)
    float2 t1 = make_float2(a0.x + C1 * b1.x + C2 * b2.x + C3 * b3.x,
                            a0.y + C1 * b1.y + C2 * b2.y + C3 * b3.y);
    float2 t2 = make_float2(a0.x + C2 * b1.x + C3 * b2.x + C1 * b3.x,
                            a0.y + C2 * b1.y + C3 * b2.y + C1 * b3.y);
    float2 t3 = make_float2(a0.x + C3 * b1.x + C1 * b2.x + C2 * b3.x,
                            a0.y + C3 * b1.y + C1 * b2.y + C2 * b3.y);
    float2 u1 = rot90<DIR>(make_float2(S1 * d1.x + S2 * d2.x + S3 * d3.x,
                                       S1 * d1.y + S2 * d2.y + S3 * d3.y));
    float2 u2 = rot90<DIR>(make_float2(S2 * d1.x - S3 * d2.x - S1 * d3.x,
                                       S2 * d1.y - S3 * d2.y - S1 * d3.y));
    float2 u3 = rot90<DIR>(make_float2(S3 * d1.x - S1 * d2.x + S2 * d3.x,
                                       S3 * d1.y - S1 * d2.y + S2 * d3.y));
    v[0] = cadd(a0, cadd(b1, cadd(b2, b3)));
    v[1] = cadd(t1, u1);
    v[6] = csub(t1, u1);
    v[2] = cadd(t2, u2);
    v[5] = csub(t2, u2);
    v[3] = cadd(t3, u3);
    v[4] = csub(t3, u3);
}

// v * W16^m for the fixed twiddles of the radix-16 codelet (c = cos, s = sin
// of 2 pi m / 16); forward multiplies by c - i s, inverse by c + i s.
template <int DIR>
__device__ __forceinline__ float2 rot16(float2 v, float c, float s) {
    return DIR < 0 ? make_float2(v.x * c + v.y * s, v.y * c - v.x * s)
                   : make_float2(v.x * c - v.y * s, v.y * c + v.x * s);
}

// Radix-16 as 4 x 4: DFT4 over n2 of a[n1 + 4 n2], twiddle W16^(n1 k2),
// DFT4 over n1; output X[k2 + 4 k1].
template <int DIR>
__device__ __forceinline__ void dft16(float2* v) {
    constexpr float c1 = 0.9238795325112867f, s1 = 0.3826834323650898f;
    constexpr float h = 0.7071067811865476f;
    float2 y[4][4];
#pragma unroll
    for (int n1 = 0; n1 < 4; ++n1) {
        float2 t[4] = {v[n1], v[n1 + 4], v[n1 + 8], v[n1 + 12]};
        dft4<DIR>(t);
#pragma unroll
        for (int k2 = 0; k2 < 4; ++k2) y[n1][k2] = t[k2];
    }
    // twiddles W16^(n1 k2), n1, k2 in 1..3: m = 1,2,3 / 2,4,6 / 3,6,9
    y[1][1] = rot16<DIR>(y[1][1], c1, s1);
    y[1][2] = rot16<DIR>(y[1][2], h, h);
    y[1][3] = rot16<DIR>(y[1][3], s1, c1);
    y[2][1] = rot16<DIR>(y[2][1], h, h);
    y[2][2] = rot90<DIR>(y[2][2]);
    y[2][3] = rot16<DIR>(y[2][3], -h, h);
    y[3][1] = rot16<DIR>(y[3][1], s1, c1);
    y[3][2] = rot16<DIR>(y[3][2], -h, h);
    y[3][3] = rot16<DIR>(y[3][3], -c1, -s1);
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) {
        float2 t[4] = {y[0][k2], y[1][k2], y[2][k2], y[3][k2]};
        dft4<DIR>(t);
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) v[k2 + 4 * k1] = t[k1];
    }
}

template <int R, int DIR>
__device__ __forceinline__ void dft(float2* v) {
    if constexpr (R == 16) dft16<DIR>(v);
    else if constexpr (R == 2) dft2<DIR>(v[0], v[1]);
    else if constexpr (R == 3) dft3<DIR>(v);
    else if constexpr (R == 4) dft4<DIR>(v);
    else if constexpr (R == 5) dft5<DIR>(v);
    else if constexpr (R == 7) dft7<DIR>(v);
    else if constexpr (R == 8) dft8<DIR>(v);
}

// One Stockham stage.  (t, jb): this thread's line and first butterfly.
template <int R, int DIR, int NS_STATIC, int SW = 0, int PPT = 32>
__device__ __forceinline__ void stage_body(float2* buf, int T, int L, int Ns_dyn, int t, int jb,
                                           int tpl, const float2* __restrict__ tw, int tws,
                                           int nin = 1 << 30, int nout = 1 << 30) {
    // nin: points >= nin are known zeros (only meaningful in a first stage,
    // where point index = input index); nout: points >= nout are not stored
    // (only in a last stage, where point index = output index).
    // ceil(PPT / R) butterflies per thread cover L / R butterflies with
    // ceil(L / PPT) threads per line for every radix (<= PPT + R - 1 values held).
    constexpr int K = (PPT + R - 1) / R;
    const int Ns = NS_STATIC > 0 ? NS_STATIC : Ns_dyn;
    const int nb = L / R;
    const int step = L / (Ns * R);  // twiddle index step in units of W_L
    float2 v[K][R];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int j = jb + k * tpl;
        if (jb < tpl && j < nb) {
#pragma unroll
            for (int r = 0; r < R; ++r)
                v[k][r] = (j + r * nb < nin) ? buf[physw<SW>(j + r * nb, t, T)] : make_float2(0.f, 0.f);
            if (Ns > 1) {
                const int kk = j % Ns;
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    const float2 w = __ldg(&tw[(r * kk * step) * tws]);
                    v[k][r] = DIR < 0 ? cmul(v[k][r], w) : cmulc(v[k][r], w);
                }
            }
            dft<R, DIR>(v[k]);
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int j = jb + k * tpl;
        if (jb < tpl && j < nb) {
            const int base = (j / Ns) * Ns * R + (j % Ns);
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (base + r * Ns < nout) buf[physw<SW>(base + r * Ns, t, T)] = v[k][r];
        }
    }
    __syncthreads();
}

// Runtime-dispatched stage for arbitrary 7-smooth lengths.  Not inlined, so
// each radix keeps its own register allocation.
template <int R, int DIR>
__device__ __noinline__ void fft_stage_dyn(float2* buf, int T, int L, int Ns, int t, int jb,
                                           int tpl, const float2* tw, int tws) {
    stage_body<R, DIR, 0, 0, kDynPPT>(buf, T, L, Ns, t, jb, tpl, tw, tws);
}

template <int DIR>
__device__ __forceinline__ void fft_lines_dyn(float2* buf, int T, int t, int jb, const Axis ax) {
    int Ns = 1;
    for (int s = 0; s < ax.nst; ++s) {
        const int R = ax.radix(s);
        switch (R) {
            case 8: fft_stage_dyn<8, DIR>(buf, T, ax.L, Ns, t, jb, ax.tpl, ax.tw, ax.tws); break;
            case 4: fft_stage_dyn<4, DIR>(buf, T, ax.L, Ns, t, jb, ax.tpl, ax.tw, ax.tws); break;
            case 2: fft_stage_dyn<2, DIR>(buf, T, ax.L, Ns, t, jb, ax.tpl, ax.tw, ax.tws); break;
            case 3: fft_stage_dyn<3, DIR>(buf, T, ax.L, Ns, t, jb, ax.tpl, ax.tw, ax.tws); break;
            case 5: fft_stage_dyn<5, DIR>(buf, T, ax.L, Ns, t, jb, ax.tpl, ax.tw, ax.tws); break;
            case 7: fft_stage_dyn<7, DIR>(buf, T, ax.L, Ns, t, jb, ax.tpl, ax.tw, ax.tws); break;
            default: break;
        }
        Ns *= R;
    }
}

// Static lengths with the radix sequence fixed at compile time
// (static_radix): straight-line stages, constant divisors for j div Ns.  The
// runtime path (plan_axis, for non-instantiated lengths) uses radices <= 8.
// The power-of-two part first, radix-16 stages first (fewest shared-memory
// round trips), then 8 / 4 / 2, then the odd factors 5 and 3:
// 64 = 16.4, 128 = 16.8, 256 = 16.16, 512 = 16.8.4, 1024 = 16.16.4,
// 80 = 16.5, 96 = 8.4.3, 160 = 8.4.5, 192 = 16.4.3, 240 = 16.5.3,
// 320 = 16.4.5, 384 = 16.8.3, 480 = 8.4.5.3, 640 = 16.8.5, 768 = 16.16.3,
// 960 = 16.4.5.3.
constexpr int static_radix(int rem) {
    const int p = rem & -rem;  // power-of-two part
    if (p > 1) return p >= 16 && p != 32 ? 16 : (p == 32 ? 8 : p);
    return rem % 5 == 0 ? 5 : (rem % 3 == 0 ? 3 : (rem % 7 == 0 ? 7 : rem));
}

template <int L, int DIR, int NS, int SW = 0>
__device__ __forceinline__ void fft_lines_static(float2* buf, int T, int t, int jb,
                                                 const float2* __restrict__ tw, int tws,
                                                 int nin = 1 << 30, int nout = 1 << 30) {
    if constexpr (NS < L) {
        constexpr int R = static_radix(L / NS);
        stage_body<R, DIR, NS, SW>(buf, T, L, NS, t, jb, (L + 31) / 32, tw, tws,
                                   NS == 1 ? nin : (1 << 30), NS * R == L ? nout : (1 << 30));
        fft_lines_static<L, DIR, NS * R, SW>(buf, T, t, jb, tw, tws, nin, nout);
    }
}

// Full transform of the T lines held in buf.  DIR = -1 forward
// (exp(-2 pi i ...)), +1 inverse, both unnormalised.  All threads of the CTA
// must call it (it contains barriers).  t = tid % T, jb = tid / T.
// LS > 0 selects the compile-time path for length LS (== ax.L).
template <int DIR, int LS>
__device__ __forceinline__ void fft_lines(float2* buf, int T, int t, int jb, const Axis ax,
                                          int nin = 1 << 30, int nout = 1 << 30) {
    if constexpr (LS > 0) {
        fft_lines_static<LS, DIR, 1>(buf, T, t, jb, ax.tw, ax.tws, nin, nout);
    } else {
        fft_lines_dyn<DIR>(buf, T, t, jb, ax);
    }
}

// Host: factor L into supported radices (order 0: 8s first, then 4/2, 5, 3,
// 7; order 1: the odd radices 5, 3, 7 first, then the power-of-two stages).
// Returns false if L has a prime factor other than 2, 3, 5, 7.
bool plan_axis(int L, Axis& ax, int order = 0);

}  // namespace dk
