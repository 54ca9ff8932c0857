// Pupil model on the device: frequency geometry, anti-aliased pupil support,
// aplanatic apodization and the Gibson-Lanni / Zernike phase aberrations.
//
// Replaces deconlib's make_geometry (psf/optics.py:96-225), make_pupil and
// aplanatic_apodization (psf/pupil.py:17-97), IndexMismatch
// (psf/aberrations/geometric.py:38-58) and ZernikeAberration
// (psf/aberrations/zernike.py:92-115 over utils/zernike.py).  All arithmetic
// is FP64, in the reference's operation order; the values that decide a
// comparison (the frequency grid, |k|, the sub-grid disc test of the support
// weight, sin / cos theta, kz) use the round-to-nearest intrinsics so no
// multiply-add is contracted, which makes them equal to NumPy's bit for bit.
// The transcendental factors (atan2, sin, cos, pow, exp) come from CUDA's FP64
// math library and agree with NumPy's to a few ulp.
//
// A pupil plane is small (ny x nx, 2-D); one thread per pixel.  Together with
// decon_pupil_to_psf this builds a job's PSF without a host round trip.
#include <cmath>
#include <vector>

#include "conv_impl.cuh"

namespace dk {

struct GeomArgs {
    int64_t ny, nx;
    double inv_y, inv_x;      // 1 / (n d) per axis: fftfreq step and sub-grid spacing
    double k_cut, k_cut_sq;   // NA / lambda and its square (host-rounded as the reference)
    double k_imm_sq;          // (ni / lambda)^2
    double wl, ni;
    int oversample;
    double sub[32];           // (j + 0.5) / oversample - 0.5
    double *kx, *ky, *kz, *rho, *phi, *support, *cos_t, *sin_t;
    uint8_t* mask;
};

__device__ __forceinline__ double fftfreq_at(int64_t i, int64_t n, double inv) {
    const int64_t half = (n - 1) / 2 + 1;  // non-negative frequencies first
    const int64_t k = i < half ? i : i - n;
    return __dmul_rn((double)k, inv);
}

__global__ void k_geometry(const __grid_constant__ GeomArgs a) {
    const int64_t n = a.ny * a.nx;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t iy = i / a.nx, ix = i - iy * a.nx;
        const double kx = fftfreq_at(ix, a.nx, a.inv_x), ky = fftfreq_at(iy, a.ny, a.inv_y);
        const double kr = __dsqrt_rn(__dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky)));
        const bool m = kr <= a.k_cut;
        double sw;
        if (a.oversample == 1) {
            sw = m ? 1.0 : 0.0;
        } else {
            int cnt = 0;
            for (int jx = 0; jx < a.oversample; ++jx) {
                const double kxs = __dadd_rn(kx, __dmul_rn(a.sub[jx], a.inv_x));
                const double kxs_sq = __dmul_rn(kxs, kxs);
                for (int jy = 0; jy < a.oversample; ++jy) {
                    const double kys = __dadd_rn(ky, __dmul_rn(a.sub[jy], a.inv_y));
                    cnt += __dadd_rn(kxs_sq, __dmul_rn(kys, kys)) <= a.k_cut_sq;
                }
            }
            sw = __ddiv_rn((double)cnt, (double)(a.oversample * a.oversample));
        }
        const double st = fmin(fmax(__ddiv_rn(__dmul_rn(a.wl, kr), a.ni), 0.0), 1.0);
        const double ct = __dsqrt_rn(__dsub_rn(1.0, __dmul_rn(st, st)));
        const double kz = __dsqrt_rn(fmax(0.0, __dsub_rn(a.k_imm_sq, __dmul_rn(kr, kr))));
        a.kx[i] = kx;
        a.ky[i] = ky;
        a.kz[i] = kz;
        a.rho[i] = m ? __ddiv_rn(kr, a.k_cut) : 0.0;
        a.phi[i] = atan2(ky, kx);
        a.mask[i] = m ? 1 : 0;
        a.support[i] = sw;
        a.cos_t[i] = ct;
        a.sin_t[i] = st;
    }
}

// Weights of the wrapped Gaussian (sigma <= 32: radius <= 128).
constexpr int kGaussMaxRadius = 128;
struct GaussW {
    int radius;
    double w[2 * kGaussMaxRadius + 1];
};

// One pass of the wrapped Gaussian along axis 0 (y) or 1 (x):
// out[l] = sum_t w[t] in[(l + t - r) mod len], clipped to [0, 1] on request.
__global__ void k_gauss_wrap(const double* __restrict__ in, double* __restrict__ out, int64_t ny,
                             int64_t nx, int axis, const __grid_constant__ GaussW g, int clip) {
    const int64_t n = ny * nx;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t iy = i / nx, ix = i - iy * nx;
        const int64_t len = axis == 0 ? ny : nx;
        const int64_t l = axis == 0 ? iy : ix;
        double acc = 0.0;
        for (int t = -g.radius; t <= g.radius; ++t) {
            int64_t s = (l + t) % len;
            if (s < 0) s += len;
            const int64_t j = axis == 0 ? s * nx + ix : iy * nx + s;
            acc = fma(g.w[t + g.radius], in[j], acc);
        }
        out[i] = clip ? fmin(fmax(acc, 0.0), 1.0) : acc;
    }
}

__global__ void k_pupil_init(const double* __restrict__ support, const double* __restrict__ cos_t,
                             const uint8_t* __restrict__ mask, int64_t n, int apodize,
                             double2* __restrict__ pupil) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        double v = support[i];
        if (apodize) {
            // pupil * (1 / sqrt(max(cos theta, eps)) * mask)
            const double c = fmax(cos_t[i], 2.220446049250313e-16);
            const double ap = __dmul_rn(__ddiv_rn(1.0, __dsqrt_rn(c)), mask[i] ? 1.0 : 0.0);
            v = __dmul_rn(v, ap);
        }
        pupil[i] = make_double2(v, 0.0);
    }
}

__device__ __forceinline__ double2 cmul_d(double2 a, double2 b) {
    return make_double2(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                        __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}

// pupil *= exp(i 2 pi depth (ns cos t2 - ni cos t1) / lambda)
__global__ void k_index_mismatch(const double* __restrict__ sin_t, const double* __restrict__ cos_t,
                                 int64_t n, double ratio, double ni, double ns, double depth,
                                 double two_pi, double wl, double2* __restrict__ pupil) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double s2 = fmin(fmax(__dmul_rn(ratio, sin_t[i]), 0.0), 1.0);
        const double c2 = __dsqrt_rn(__dsub_rn(1.0, __dmul_rn(s2, s2)));
        const double opd = __dmul_rn(depth, __dsub_rn(__dmul_rn(ns, c2), __dmul_rn(ni, cos_t[i])));
        const double ph = __ddiv_rn(__dmul_rn(two_pi, opd), wl);
        double sn, cs;
        sincos(ph, &sn, &cs);
        pupil[i] = cmul_d(pupil[i], make_double2(cs, sn));
    }
}

// pupil *= exp(2 pi i kz z): ((2 pi) kz) z as the reference forms it
__global__ void k_defocus(const double* __restrict__ kz, int64_t n, double two_pi, double z,
                          double2* __restrict__ pupil) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double ph = __dmul_rn(__dmul_rn(two_pi, kz[i]), z);
        double sn, cs;
        sincos(ph, &sn, &cs);
        pupil[i] = cmul_d(pupil[i], make_double2(cs, sn));
    }
}

constexpr int kZernMaxTerms = 32, kZernMaxRadial = 10;

struct ZernTerm {
    int m, nrad;
    double coef, norm;
    double rc[kZernMaxRadial];
    int pw[kZernMaxRadial];
};

struct ZernArgs {
    int nterms;
    ZernTerm t[kZernMaxTerms];
};

// pupil *= exp(i mask sum_j c_j Z_j(rho, phi)); the sum in the terms' order
__global__ void k_zernike(const __grid_constant__ ZernArgs a, const double* __restrict__ rho,
                          const double* __restrict__ phi, const uint8_t* __restrict__ mask,
                          int64_t n, double2* __restrict__ pupil) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double r = rho[i], p = phi[i];
        double phase = 0.0;
        for (int j = 0; j < a.nterms; ++j) {
            const ZernTerm& t = a.t[j];
            double R = 0.0;
            for (int k = 0; k < t.nrad; ++k) R = __dadd_rn(R, __dmul_rn(t.rc[k], t.pw[k] == 0 ? 1.0 : pow(r, (double)t.pw[k])));
            const int am = t.m < 0 ? -t.m : t.m;
            const double ang = t.m >= 0 ? cos(__dmul_rn((double)t.m, p)) : sin(__dmul_rn((double)am, p));
            const double z = t.m >= 0 ? __dmul_rn(__dmul_rn(t.norm, R), ang)
                                      : __dmul_rn(__dmul_rn(-t.norm, R), ang);
            phase = __dadd_rn(phase, __dmul_rn(t.coef, z));
        }
        phase = __dmul_rn(phase, mask[i] ? 1.0 : 0.0);
        double sn, cs;
        sincos(phase, &sn, &cs);
        pupil[i] = cmul_d(pupil[i], make_double2(cs, sn));
    }
}

static int grid_1d(int64_t n) {
    return (int)std::max<int64_t>(1, std::min<int64_t>(cdiv(n, 256), (int64_t)sm_count() * 8));
}

}  // namespace dk

using namespace dk;

extern "C" {

int decon_psf_geometry(int64_t ny, int64_t nx, double dy, double dx, double wavelength, double na,
                       double ni, int oversample, double smoothing_sigma, double* kx, double* ky,
                       double* kz, double* rho, double* phi, uint8_t* mask, double* support,
                       double* cos_theta, double* sin_theta, double* scratch, void* stream) {
    if (!kx || !ky || !kz || !rho || !phi || !mask || !support || !cos_theta || !sin_theta)
        return fail(DECON_ERR_NULL, "decon_psf_geometry: null pointer");
    if (ny < 1 || nx < 1) return fail(DECON_ERR_VALUE, "shape must be positive");
    if (!(dy > 0) || !(dx > 0)) return fail(DECON_ERR_VALUE, "Spacing must be positive, got (%g, %g)", dy, dx);
    if (oversample < 1 || oversample > 32)
        return fail(DECON_ERR_VALUE, "oversample must be in [1, 32], got %d", oversample);
    if (smoothing_sigma < 0)
        return fail(DECON_ERR_VALUE, "boundary_smoothing_sigma must be >= 0, got %g", smoothing_sigma);
    if (smoothing_sigma > 0 && !scratch)
        return fail(DECON_ERR_NULL, "decon_psf_geometry: smoothing needs an ny * nx scratch");
    GeomArgs a{};
    a.ny = ny;
    a.nx = nx;
    a.inv_y = 1.0 / ((double)ny * dy);
    a.inv_x = 1.0 / ((double)nx * dx);
    a.k_cut = na / wavelength;
    a.k_cut_sq = a.k_cut * a.k_cut;
    const double k_imm = ni / wavelength;
    a.k_imm_sq = k_imm * k_imm;
    a.wl = wavelength;
    a.ni = ni;
    a.oversample = oversample;
    for (int j = 0; j < oversample; ++j) a.sub[j] = ((double)j + 0.5) / (double)oversample - 0.5;
    a.kx = kx;
    a.ky = ky;
    a.kz = kz;
    a.rho = rho;
    a.phi = phi;
    a.support = support;
    a.cos_t = cos_theta;
    a.sin_t = sin_theta;
    a.mask = mask;
    const cudaStream_t st = as_stream(stream);
    const int64_t n = ny * nx;
    k_geometry<<<grid_1d(n), 256, 0, st>>>(a);
    DK_LAUNCHED();
    if (smoothing_sigma > 0) {
        // scipy.ndimage.gaussian_filter, mode "wrap", truncate 4: radius
        // int(4 sigma + 0.5), weights exp(-x^2 / (2 sigma^2)) / sum, axis 0 then 1
        GaussW g{};
        g.radius = (int)(4.0 * smoothing_sigma + 0.5);
        if (g.radius > kGaussMaxRadius)
            return fail(DECON_ERR_UNSUPPORTED, "boundary_smoothing_sigma %g > 32", smoothing_sigma);
        double sum = 0.0;
        for (int t = -g.radius; t <= g.radius; ++t) {
            g.w[t + g.radius] = std::exp(-0.5 / (smoothing_sigma * smoothing_sigma) * (double)(t * t));
            sum += g.w[t + g.radius];
        }
        for (int t = 0; t <= 2 * g.radius; ++t) g.w[t] /= sum;
        k_gauss_wrap<<<grid_1d(n), 256, 0, st>>>(support, scratch, ny, nx, 0, g, 0);
        DK_LAUNCHED();
        k_gauss_wrap<<<grid_1d(n), 256, 0, st>>>(scratch, support, ny, nx, 1, g, 1);
        DK_LAUNCHED();
    }
    return DECON_OK;
}

int decon_psf_pupil(const double* support, const double* cos_theta, const uint8_t* mask, int64_t n,
                    int apodize, double* pupil, void* stream) {
    if (!support || !pupil || (apodize && (!cos_theta || !mask)))
        return fail(DECON_ERR_NULL, "decon_psf_pupil: null pointer");
    k_pupil_init<<<grid_1d(n), 256, 0, as_stream(stream)>>>(support, cos_theta, mask, n, apodize,
                                                             reinterpret_cast<double2*>(pupil));
    DK_LAUNCHED();
    return DECON_OK;
}

int decon_psf_index_mismatch(const double* sin_theta, const double* cos_theta, int64_t n,
                             double wavelength, double ni, double ns, double depth, double* pupil,
                             void* stream) {
    if (!sin_theta || !cos_theta || !pupil) return fail(DECON_ERR_NULL, "decon_psf_index_mismatch: null pointer");
    if (!(ns > 0) || !(wavelength > 0)) return fail(DECON_ERR_VALUE, "ns and wavelength must be positive");
    k_index_mismatch<<<grid_1d(n), 256, 0, as_stream(stream)>>>(sin_theta, cos_theta, n, ni / ns, ni, ns,
                                                                 depth, 2.0 * M_PI, wavelength,
                                                                 reinterpret_cast<double2*>(pupil));
    DK_LAUNCHED();
    return DECON_OK;
}

int decon_psf_defocus(const double* kz, int64_t n, double z, double* pupil, void* stream) {
    if (!kz || !pupil) return fail(DECON_ERR_NULL, "decon_psf_defocus: null pointer");
    k_defocus<<<grid_1d(n), 256, 0, as_stream(stream)>>>(kz, n, 2.0 * M_PI, z,
                                                          reinterpret_cast<double2*>(pupil));
    DK_LAUNCHED();
    return DECON_OK;
}

static uint64_t fact(int k) {
    uint64_t f = 1;
    for (int i = 2; i <= k; ++i) f *= (uint64_t)i;
    return f;
}

int decon_psf_zernike(const double* rho, const double* phi, const uint8_t* mask, int64_t n,
                      int nterms, const int* j, const double* coef, double* pupil, void* stream) {
    if (!rho || !phi || !mask || !pupil || (nterms > 0 && (!j || !coef)))
        return fail(DECON_ERR_NULL, "decon_psf_zernike: null pointer");
    ZernArgs a{};
    int used = 0;
    for (int q = 0; q < nterms; ++q) {
        if (coef[q] == 0.0) continue;
        if (used == kZernMaxTerms)
            return fail(DECON_ERR_UNSUPPORTED, "at most %d non-zero Zernike terms", kZernMaxTerms);
        if (j[q] < 0) return fail(DECON_ERR_VALUE, "Zernike index must be >= 0, got %d", j[q]);
        // OSA/ANSI j -> (n, m) (utils/zernike.py ansi_to_nm)
        const int nn = (int)std::ceil((-3.0 + std::sqrt(9.0 + 8.0 * j[q])) / 2.0);
        const int m = 2 * j[q] - nn * (nn + 2);
        if (nn > 18) return fail(DECON_ERR_UNSUPPORTED, "Zernike radial order %d > 18", nn);
        const int am = m < 0 ? -m : m;
        ZernTerm& t = a.t[used++];
        t.m = m;
        t.coef = coef[q];
        t.norm = std::sqrt(2.0 * (nn + 1) / (1.0 + (m == 0 ? 1.0 : 0.0)));
        t.nrad = (nn - am) / 2 + 1;
        for (int k = 0; k < t.nrad; ++k) {
            // (-1)^k (n - k)! / (k! ((n + m) / 2 - k)! ((n - m) / 2 - k)!): integers
            // below 2^53, so the quotient is the correctly rounded one
            const double num = (double)fact(nn - k);
            const double den = (double)(fact(k) * fact((nn + am) / 2 - k) * fact((nn - am) / 2 - k));
            t.rc[k] = (k % 2 ? -1.0 : 1.0) * (num / den);
            t.pw[k] = nn - 2 * k;
        }
    }
    a.nterms = used;
    if (used == 0) return DECON_OK;  // exp(i 0) = 1
    k_zernike<<<grid_1d(n), 256, 0, as_stream(stream)>>>(a, rho, phi, mask, n,
                                                          reinterpret_cast<double2*>(pupil));
    DK_LAUNCHED();
    return DECON_OK;
}

}  // extern "C"
