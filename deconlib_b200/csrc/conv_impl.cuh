// Internal declarations of the convolution passes (conv.cu) shared with the
// C ABI (capi.cu) and the solver kernels.
#pragma once

#include <cuda.h>
#include <cuda_fp16.h>

#include "common.cuh"
#include "fft_engine.cuh"

namespace dk {

constexpr int kSmemElems = 8192;  // complex values per CTA (64 KB)
// T lines x L points <= kSmemElems and ceil(L/32) threads per line bound a
// CTA to kSmemElems / 32 threads.
constexpr int kFftThreads = kSmemElems / 32;

// Lines per CTA for an axis: the largest power of two <= cap whose tile fits
// kSmemElems complex values and whose threads (T x tpl) fit the CTA limit of
// the length's path.
inline int fft_lines_per_cta(const Axis& ax, int cap) {
    const int lim = static_length(ax.L) ? kFftThreads : kDynThreads;
    int T = 1;
    while (T * 2 <= cap && (T * 2) * ax.L <= kSmemElems && (T * 2) * ax.tpl <= lim) T *= 2;
    return T;
}

// A float32 array of shape (wz, wy, wx) placed at offset (oz, oy, ox) inside
// the N-space volume; voxels outside the box read as zero / are not written.
struct Win3 {
    int64_t wz, wy, wx;
    int64_t oz, oy, ox;
};

inline Win3 full_window(const int64_t* N) { return Win3{N[0], N[1], N[2], 0, 0, 0}; }

// PRO_UP2: the input is the coarse (Nz/2, Ny/2, Nx/2) array of a 2x fractional-area
// downsample and the X pass reads its adjoint (every fine voxel takes its
// coarse voxel's value).  EPI_DOWN2: the output is the 2x area sum of the
// convolved volume, written at the coarse shape.
enum Prologue { PRO_ARRAY = 0, PRO_CONST = 1, PRO_KERNEL = 2, PRO_RLINIT = 3, PRO_UP2 = 4 };
enum Epilogue { EPI_STORE = 0, EPI_RL_RATIO = 1, EPI_RL_UPDATE = 2, EPI_PRED = 3, EPI_DOWN2 = 4 };
enum ColMode { COL_FWD = 0, COL_INV = 1, COL_OTF = 2, COL_OTF_CONJ = 3 };
// kernel classes for decon_profile_start (bit mask)
enum ProfClass { PROF_XR2C = 1, PROF_COL = 2, PROF_ZOTF = 4, PROF_XC2R = 8 };

struct XR2CArgs {
    const float* in;
    float cval, bg, kdiv;
    int64_t Nz, Ny, Nx;  // rows = Nz * Ny, row length Nx (zero-padded to Fx)
    Win3 win;
    int64_t Kz, Ky, Kx, pz, py, px;  // kernel embedding (PRO_KERNEL)
    float2* out;
    int64_t P, nrows;
    int Hx, odd, T, vec4;
    Axis ax;            // length Fx/2 (even Fx) or Fx (odd)
    const float2* twx;  // W_Fx table
    FastDiv fd_q4, fd_H, fd_nin, fd_np;  // Nx / 4, Hx, packed non-zero points, L / 2 + 1
    // 0: spectrum rows of pitch P (element (row, kx) at row * P + kx); > 0:
    // kx-major spectrum, element (row, kx) at kx * kstride + row (kstride =
    // Nz * Ny), the layout of the fused Y / axial pass
    int64_t kstride;
};

struct ColArgs {
    const float2* src;
    float2* dst;
    int64_t src_os, src_js, dst_os, dst_js;
    int nin, nout, ncols, T, mode, ntiles;
    Axis ax;
    const float2* otf;
    int64_t otf_js, otf_os;
};

struct ColTmaArgs {
    CUtensorMap src, dst, otf;  // 64-byte aligned descriptors
    int nin, nout, ntiles, mode;
    int src_jdim, dst_jdim, src_box, dst_box, otf_box;
    int tws;
    const float2* tw;
};

// Persistent pipelined column pass (k_col_pipe).
struct PipeArgs {
    CUtensorMap src, dst;
    CUtensorMap otfmap;     // FP32 OTF [Fz][Fy][P] as TMA boxes (axial pass)
    CUtensorMap otfmap16;   // FP16 OTF [Fz][Fy][P] half2, (16, 1, otf_box) boxes (lean mixed axial pass)
    int otf_box;
    const float2* otf;      // OTF base for the axial pass
    const __half2* otf16;   // mixed precision: FP16 OTF, OTF = otf16 * otf_inv[kz]
    const float* otf_inv;
    int64_t otf_js, otf_os; // complex-element strides of OTF rows (kz) and planes (ky)
    const float2* tw;       // W_L table, W_L^m = tw[m * tws]
    int tws;
    int nin, nout, ntiles, nouter;
    int src_jdim, dst_jdim, src_box, dst_box;
};

struct XC2RArgs {
    const float2* in;
    int64_t P, Ny, Nx, nrows;
    int Hx, odd, T, vec4;
    Axis ax;
    const float2* twx;
    float scale;
    Win3 win;
    float* out;
    const float* aux0;
    const float* aux1;
    float bg;
    double* partials;
    FastDiv fd_L, fd_h2, fd_npair, fd_q4, fd_Nx;  // L, L / 2, L / 2 + 1, Nx / 4, Nx
    int64_t kstride;  // as XR2CArgs::kstride
};

// Device-resident state of one LinearFFTConvolver.
struct ConvPlan {
    int64_t N[3], F[3], K[3];
    int64_t Hx, P;
    int odd;
    Axis ax_x, ax_y, ax_z;
    int T_x, T_y, T_z;
    float2 *otf, *s1, *s2;
    float2 *twx, *twy, *twz;
    double* dscal;        // device scalars (kernel sum, reductions)
    double* partials;     // per-CTA FP64 partial sums of fused reductions
    int64_t npartials;
    float kdiv;
    double norm_sq;
    int device;
    // TMA descriptors of the column passes (valid when tma_y / tma_z)
    bool tma_y = false, tma_z = false;
    CUtensorMap tm_s1_j1, tm_s2_j1, tm_s2_j2, tm_otf_z;
    int s1_box = 0, s2y_box = 0, s2z_box = 0, otf_box = 0;
    // Mixed precision (decon_conv_set_precision): the OTF also stored as FP16
    // complex, scaled per kz plane by a power of two (OTF = otf16 * otf_inv[kz]),
    // read by the pipelined axial pass instead of the FP32 OTF.
    int precision = 0;
    __half2* otf16 = nullptr;
    float* otf_inv = nullptr;
    CUtensorMap tm_otf16_z;   // valid when tma_otf16
    bool tma_otf16 = false;
    // Fused Y / axial pass (yzpass.cuh): the OTF also stored kx-major
    // [Hx][Fy][Fz]; the spectrum between the X passes is then kx-major too
    // ([Hx][Nz][Ny] in s1).  nullptr: the canvas takes the unfused passes.
    float2* otft = nullptr;
    // Schedule (decon_conv_set_schedule): DECON_SCHED_* bits choosing among
    // equivalent pass families; T*_0 / ax*_0 keep the default lines per CTA
    // and radix plans the schedule modifies.
    int sched = 0;
    int T_x0 = 0, T_y0 = 0, T_z0 = 0;
};

// Canvas and signal extents the fused Y / axial pass implements (Fy in {256,
// 512}, Fz in {128, 256}, the signal in the first half of both axes, Ny even).
bool yz_supported(const int64_t N[3], const int64_t F[3]);
// True when this plan's convolutions run the fused Y / axial pass.
bool use_yz(const ConvPlan& p);
// Fill p.otft from p.otf (after every OTF build).
int build_otf_kmajor(const ConvPlan& p, cudaStream_t st);

// Quantise p.otf into p.otf16 / p.otf_inv (capi.cu).
int quantize_otf(const ConvPlan& p, cudaStream_t st);
// True when the axial pass of this plan runs the pipelined kernel (conv.cu).
bool zpass_pipelined(const ConvPlan& p);

// Shared-memory opt-in (only ever raised per device and kernel) and cached
// occupancy for a launch shape (conv.cu).
int kernel_prepare(void* fn, size_t smem, int nthr, int* per_sm);

bool tma_length_ok(int L);
// Kernels of the X R2C / X C2R / plain column passes for one axis length
// (the static-length instantiation, or the runtime-radix one), by prologue /
// epilogue code; nullptr for an unknown code.  One translation unit each
// (xstatic_r2c.cu, xstatic_c2r.cu, xstatic_col.cu), so they build in parallel.
void* pick_xr2c_kernel(int pro, int L);
void* pick_xc2r_kernel(int epi, int L);
void* pick_colfft_kernel(int L);

// Rank-3 map over an FP16 complex [d2][d1][pitch] buffer (one half2 = one
// 4-byte element) with (16, 1, b2) boxes and no swizzle.
bool encode_half_plane_map(CUtensorMap* map, const __half2* base, int64_t pitch, int64_t d1, int64_t d2,
                           int b2);
bool encode_spectrum_map(CUtensorMap* map, const float2* base, int64_t pitch, int64_t d1, int64_t d2,
                         int b1, int b2);

int launch_xr2c(const ConvPlan& p, int pro, const float* in, Win3 win, float cval, float bg,
                int64_t nz_rows, float2* out, cudaStream_t st, int64_t kstride = 0);
int launch_col(const ConvPlan& p, const Axis& ax, int T, int mode, const float2* src,
               int64_t src_os, int64_t src_js, int nin, float2* dst, int64_t dst_os,
               int64_t dst_js, int nout, int64_t nouter, cudaStream_t st);
int launch_xc2r(const ConvPlan& p, int epi, const float2* in, Win3 win, float* out,
                const float* aux0, const float* aux1, float bg, double* partials, int* nblk_out,
                cudaStream_t st);
int spectrum_forward(const ConvPlan& p, int pro, const float* in, Win3 win, float cval, float bg,
                     cudaStream_t st);
int spectrum_filter_back(const ConvPlan& p, bool adjoint, cudaStream_t st);

// FP64 reductions (reduce.cu)
int reduce_f32(const float* a, const float* b, int64_t n, int op, double* out, double* partials,
               int64_t npartials, cudaStream_t st);
int finish_partials(const double* partials, int n, double* out, cudaStream_t st);
int64_t reduce_partials_needed();

}  // namespace dk

struct decon_conv : dk::ConvPlan {};
