/*
 * decon_b200.h -- C ABI of the B200 (sm_100a) 3D deconvolution library.
 *
 * The library is the device side of deconlib's deconvolution hot path:
 * linear FFT convolution, pad/crop, fractional-area resampling, Hessian and
 * gradient stencils, Richardson-Lucy and adaptive-PDHG iterations.  Every
 * entry point takes plain pointers, int64 shapes and a CUDA stream passed as
 * ``void*`` (a ``cudaStream_t``; NULL is the legacy default stream).  Array
 * pointers are DEVICE pointers to C-contiguous float32 data unless the
 * comment says "host".  Volumes are (z, y, x); 1-D and 2-D problems are
 * passed with leading extents of 1.
 *
 * Every function returns a status code (DECON_OK == 0).  On failure
 * decon_last_error() returns a message for the calling host thread.  Launches
 * are asynchronous: a status of DECON_OK means the work was queued.  Only the
 * functions documented as "synchronises" wait for the device.
 *
 * The reference (deconlib 0.4.0) is pure Python on MLX; it has no native
 * FFI.  Each entry point below names the Python interface it replaces
 * (file:line inside the deconlib project).
 */
#ifndef DECON_B200_H
#define DECON_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define DECON_OK 0
#define DECON_ERR_VALUE 1       /* bad shape or argument (Python: ValueError) */
#define DECON_ERR_UNSUPPORTED 2 /* size the kernels do not implement            */
#define DECON_ERR_OOM 3         /* device allocation failed                    */
#define DECON_ERR_CUDA 4        /* CUDA runtime error                          */
#define DECON_ERR_TIMEOUT 5     /* a bounded device wait ran out               */
#define DECON_ERR_NULL 6        /* null handle or pointer                      */

/* Message for the last failing call on this host thread ("" if none). */
const char* decon_last_error(void);
/* Library ABI version (major * 10000 + minor * 100 + patch). */
int decon_version(void);
/* Synchronises the stream and reports DECON_ERR_TIMEOUT if any kernel's
 * bounded TMA/mbarrier wait gave up since load or since the last
 * decon_device_status_clear (the results of that kernel are invalid). */
int decon_device_status(void* stream);
/* Synchronises the stream and clears the timeout record that
 * decon_device_status reads, so later checks report only new timeouts. */
int decon_device_status_clear(void* stream);
/* Test hook for the bounded waits (no counterpart in the reference): one
 * CTA waits, through the same bounded mbarrier wait the TMA kernels use, on
 * a barrier that nothing completes; after `polls` polls (1..65536) the wait
 * gives up, records the timeout and the kernel returns.  Faults nothing and
 * leaves the context usable; decon_device_status then reports
 * DECON_ERR_TIMEOUT until decon_device_status_clear. */
int decon_test_wait_timeout(unsigned polls, void* stream);
/* Kernels launched by this library since load (benchmark accounting). */
int64_t decon_launch_count(void);

/* ---- FFT sizing (deconvolution/linops_mlx.py:956-1032) ---------------- */

/* Smallest m >= n whose prime factors are 2, 3 and 5 only
 * (linops_mlx.py:956 _next_smooth_number). */
int64_t decon_next_smooth(int64_t n);

/* Per-axis 5-smooth canvas >= max(N + pad, M); pad_or_minus1[i] < 0 means
 * the default M - 1 (linops_mlx.py:975 fast_padded_shape).  Host arrays. */
int decon_fast_padded_shape(int ndim, const int64_t* signal, const int64_t* kernel,
                            const int64_t* pad_or_minus1, int64_t* out);

/* ---- linear FFT convolution (deconvolution/linops_mlx.py:435-533) ------ */

typedef struct decon_conv decon_conv; /* opaque plan: OTF, spectra, twiddles */

/* LinearFFTConvolver.__init__ (linops_mlx.py:473-518): embeds the
 * corner-origin kernel (utils/padding.py:142) in the canvas fft_shape,
 * divides by its sum when normalize != 0 (FP64 sum) and stores
 * OTF = rfftn(kernel) resident on the device.  kernel: device, shape kshape.
 * Validates fft_shape >= signal + kernel - 1 (DECON_ERR_VALUE otherwise).
 * Synchronises (the plan is ready on return). */
int decon_conv_create(const float* kernel, const int64_t kshape[3], const int64_t signal_shape[3],
                      const int64_t fft_shape[3], int normalize, void* stream, decon_conv** out);
/* FFTConvolver.__init__ (linops_mlx.py:395-415): circular convolution on the
 * kernel's own shape (canvas = signal = kernel shape, no corner embedding).
 * Synchronises. */
int decon_conv_create_circular(const float* kernel, const int64_t shape[3], int normalize,
                               void* stream, decon_conv** out);
/* Rebuild the OTF of an existing plan for a new kernel of the same kernel
 * shape (same normalisation rule, operator_norm_sq recomputed), reusing its
 * device buffers: no cudaMalloc / cudaFree, so a serving loop can hand a
 * pooled plan to the next job of the same shape without the device-wide
 * synchronisation of cudaFree.  Queued on `stream`, which it synchronises
 * (the two FP64 scalars are read back).  Replaces constructing a new
 * FFTConvolver (linops_mlx.py:395-415) for a same-shape kernel. */
int decon_conv_set_kernel(decon_conv* plan, const float* kernel, int normalize, void* stream);
/* Storage precision of the OTF read by the axial pass.  0: FP32 (default).
 * 1 (mixed): the OTF is also kept as FP16 complex with a power-of-two scale
 * per kz plane (max |OTF| of the plane maps below 2^14, so no plane loses
 * range), and the pipelined axial pass reads it (half the OTF bytes);
 * transforms, products and all reductions stay FP32 / FP64.  Needs the
 * pipelined axial pass (DECON_ERR_UNSUPPORTED otherwise).  decon_conv_set_kernel
 * requantises.  No reference counterpart: deconlib computes in the FP32 /
 * complex64 of its arrays (linops_mlx.py:411-429). */
int decon_conv_set_precision(decon_conv* plan, int precision, void* stream);
int decon_conv_destroy(decon_conv* plan);
/* operator_norm_sq = max |OTF|^2 (linops_mlx.py:415). */
int decon_conv_norm_sq(const decon_conv* plan, double* out);
/* Schedules: equivalent pass families of one plan, chosen by an autotuner
 * (no reference counterpart; results agree to FP32 rounding, 1e-6).  Bits:
 *   FUSED        the fused Y / axial cluster pass where the canvas allows it
 *                (allocates the kx-major OTF copy on first request; DECON_YZ=1
 *                selects it for every plan)
 *   NO_PIPE      one-tile TMA column kernels instead of the persistent pipelined ones
 *   NO_TMA       plain-load column kernels (no tensor maps)
 *   LEAN_OFF     one-CTA-per-SM axial kernel instead of the two-CTA (lean) one
 *   ODD_RADIX    radix plans with the 5 / 3 / 7 stages first (runtime-length axes)
 *   HALF_LINES   half the lines per CTA on runtime-length axes (more, smaller CTAs) */
#define DECON_SCHED_FUSED 1
#define DECON_SCHED_NO_PIPE 2
#define DECON_SCHED_NO_TMA 4
#define DECON_SCHED_LEAN_OFF 8
#define DECON_SCHED_ODD_RADIX 16
#define DECON_SCHED_HALF_LINES 32
int decon_conv_set_schedule(decon_conv* plan, int sched);
int decon_conv_get_schedule(const decon_conv* plan, int* sched);
/* 1 when this plan's convolutions run the fused Y / axial pass (opt-in; one
 * thread-block cluster per kx column; canvases with Fy in {256, 512}, Fz in
 * {128, 256}, the signal in the first half of both axes, even Ny, FP32 OTF),
 * 0 when they run the separate Y and axial passes.  No reference
 * counterpart (a property of this implementation). */
int decon_conv_fused_yz(const decon_conv* plan, int* out);
/* Canvas fft_shape and the spectrum row pitch (complex elements). Host. */
int decon_conv_shape(const decon_conv* plan, int64_t fft_shape[3], int64_t* pitch);
/* Copies the OTF (fft_z, fft_y, fft_x/2+1) complex64 into out (device). */
int decon_conv_get_otf(const decon_conv* plan, float* out_interleaved, void* stream);

/* LinearFFTConvolver.forward: zero-pad, circular convolution, crop
 * (linops_mlx.py:520-524).  x, y: signal_shape; y may alias x. */
int decon_conv_forward(decon_conv* plan, const float* x, float* y, void* stream);
/* LinearFFTConvolver.adjoint: correlation with conj(OTF)
 * (linops_mlx.py:526-530). */
int decon_conv_adjoint(decon_conv* plan, const float* y, float* x, void* stream);
/* compose(FractionalAreaDownsample(2), LinearFFTConvolver) (composition.py:92-106
 * over core_operators.py:222-352 and linops_mlx.py:520-530) when the
 * downsample halves every axis exactly (n_large = 2 n_small): forward writes
 * the coarse (Nz/2, Ny/2, Nx/2) 2x area sum of the convolution straight from
 * the last FFT pass; adjoint takes the coarse array and convolves its
 * adjoint (each fine voxel = its coarse voxel) read in the first FFT pass.
 * Same float32 values as the operator-by-operator path (unit weights, the
 * passes' summation order).  DECON_ERR_UNSUPPORTED unless N and Fx are even
 * (and Ny a multiple of the X pass's half line count). */
int decon_conv_forward_down2(decon_conv* plan, const float* x, float* y_coarse, void* stream);
int decon_conv_adjoint_up2(decon_conv* plan, const float* y_coarse, float* x, void* stream);

/* ---- Richardson-Lucy fused iterations (deconvolution/rl_mlx.py:83-185) - */

/* RL set-up (rl_mlx.py:122-133): sens_raw = A^T 1, floor = max(max(sens)
 * 1e-6, 1e-10); writes sens_masked = sens where sens > floor else 0 and
 * x = active ? max(x_init, 1e-6) : 0.  If x_init is NULL, x0 = A^T max(y - b,
 * 1e-6) as the reference does.  All arrays signal_shape.  Synchronises. */
int decon_rl_setup(decon_conv* plan, const float* observed, float background, const float* x_init,
                   float* x, float* sens_masked, void* stream);
/* One RL iteration for blur_op = LinearFFTConvolver (rl_mlx.py:146-150):
 * ratio = y / max(A x + b, 1e-10) fused into the forward pass epilogue and
 * x = max(x * (sens>0 ? A^T ratio / sens : 0), 1e-10) fused into the adjoint
 * pass epilogue.  ratio is caller scratch (signal_shape).  If loss_partials
 * is non-NULL, the forward epilogue also accumulates the Poisson
 * I-divergence of the INCOMING x (rl_mlx.py:58-80) into
 * loss_partials[0] as an FP64 sum (see decon_rl_loss_finish). */
int decon_rl_iteration(decon_conv* plan, const float* observed, float background,
                       const float* sens_masked, float* x, float* ratio, double* loss_sum,
                       void* stream);
/* pred = A x + b and (if loss_sum != NULL) the FP64 I-divergence sum of
 * (observed, pred) (rl_mlx.py:159-160,174). */
int decon_rl_predict(decon_conv* plan, const float* observed, float background, const float* x,
                     float* pred, double* loss_sum, void* stream);
/* `iterations` RL iterations queued back to back with no host
 * synchronisation and no loss (graph-capturable): the loop body of
 * rl_mlx.py:140-152 `iterations` times. */
int decon_rl_run(decon_conv* plan, const float* observed, float background, const float* sens,
                 float* x, float* ratio, int iterations, void* stream);

/* ---- nonlinear conjugate gradients (deconvolution/nlcg_mlx.py:326-545) ----
 * The passes of nlcg_with_operator other than the caller's operators (the
 * convolutions and the regulariser): each is one fused elementwise kernel
 * with deterministic FP64 sums kept in the handle's device scalars.  The
 * Newton-Raphson step length (nlcg_step_length, :197-300) runs on the device
 * (decon_nlcg_newton); decon_nlcg_read is the one synchronising call.  All
 * arrays are device float32; "data" arrays have the observation's size nd,
 * "object" arrays the reconstruction's size no.  eps is the reference's 1e-10. */
typedef struct decon_nlcg decon_nlcg;
int decon_nlcg_create(decon_nlcg** out);
int decon_nlcg_destroy(decon_nlcg* h);
/* s = sqrt(max(x, 1e-6)), f = s^2 (:431-439); from_s != 0: f = x^2 only. */
int decon_nlcg_init(const float* x, float* s, float* f, int64_t n, int from_s, void* stream);
/* w = 1 - g / max(m, eps) (w may be NULL) and the data sums of model m. */
int decon_nlcg_model(decon_nlcg* h, const float* m, const float* g, float eps, float* w, int64_t n,
                     void* stream);
/* mode 0: direction d; mode 1: d_out = r + gamma d (:517).  sd = s d, dd = d^2.
 * Resets the device step length to 0. */
int decon_nlcg_products(decon_nlcg* h, int mode, float gamma, const float* s, const float* d,
                        const float* r, float* d_out, float* sd, float* dd, int64_t n, void* stream);
/* Gram matrix of the regulariser images C f, C(s d), C(d^2) (n values each). */
int decon_nlcg_gram(decon_nlcg* h, const float* a, const float* b, const float* c, int64_t n,
                    void* stream);
/* newton_iters refinements of the step length (:262-291); the regulariser
 * terms come from the Gram entries when use_reg != 0. */
int decon_nlcg_newton(decon_nlcg* h, const float* m, const float* ksd, const float* kdd, const float* g,
                      float background, float eps, double beta, int use_reg, int newton_iters,
                      int64_t n, void* stream);
/* m_new = (m - b) + 2 lam K(sd) + lam^2 K(dd) + b (:297), w_new and the data
 * sums; with s != NULL also s_new = s + lam d, f_new = s_new^2 (:398-399). */
int decon_nlcg_accept(decon_nlcg* h, const float* m, const float* ksd, const float* kdd, const float* g,
                      float background, float eps, float* m_new, float* w_new, int64_t nd,
                      const float* s, const float* d, float* s_new, float* f_new, int64_t no,
                      void* stream);
/* sum a^2 (the regulariser energy ||C f||^2). */
int decon_nlcg_energy(decon_nlcg* h, const float* a, int64_t n, void* stream);
/* r = -(2 s ktw + c4b s ctcf) (ctcf may be NULL; c4b = 4 beta) and sum r^2
 * (ktw NULL: no gradient), sum f and, with f_prev, the I-divergence between
 * f_prev and f (:303-323). */
int decon_nlcg_gradient(decon_nlcg* h, const float* s, const float* f, const float* f_prev,
                        const float* ktw, const float* ctcf, float c4b, float eps, float* r, int64_t n,
                        void* stream);
/* Hessian3D regulariser (spacing ratio r) evaluated on the fly, its images
 * never stored: the Gram matrix of H f, H(s d), H(d^2) (replaces
 * decon_nlcg_gram on materialised images) and ||H f||^2 (decon_nlcg_energy).
 * shape = (nz, ny, nx) of the object arrays. */
int decon_nlcg_hess_gram(decon_nlcg* h, const float* f, const float* sd, const float* dd,
                         const int64_t shape[3], float r, void* stream);
int decon_nlcg_hess_energy(decon_nlcg* h, const float* f, const int64_t shape[3], float r, void* stream);
/* sum (g / max(m^2, eps)) ksd^2 and sum a d^2 (nlcg_hessian_quadform, :181-193). */
int decon_nlcg_quad(decon_nlcg* h, const float* g, const float* m, const float* ksd, int64_t nd,
                    const float* a, const float* d, int64_t no, float eps, void* stream);
/* Synchronise and read the 18 scalars: lam, Newton stopped, refinements run,
 * data sums [3], regulariser energy, sum r^2, I-divergence, sum f, quadratic
 * sums [2], Gram entries [6]. */
int decon_nlcg_read(decon_nlcg* h, double* out, void* stream);

/* ---- PSF synthesis (psf/widefield.py:18-73 pupil_to_psf) -----------------
 * psf[z][y][x] = |IFFT2(pupil * exp(2 pi i kz z_z))|^2 for nz planes, on the
 * device: pupil complex64 [ny][nx] (interleaved floats, DC at the corner),
 * kz float64 [ny][nx], z float64 [nz], psf float32 [nz][ny][nx] (all device
 * pointers).  normalize != 0 scales to unit sum (total from Parseval:
 * nz ny nx sum|pupil|^2, in FP64), else applies numpy's ifft2 factor
 * 1 / (ny nx)^2.  ny, nx <= 8192 and 7-smooth.  Stream-ordered: the inputs
 * must stay valid until the work on `stream` completes; complex scratch of at
 * most 256 MB (or one plane) comes from a library-owned stream-ordered pool.
 * The first call for an axis length uploads its twiddle table synchronously. */
int decon_pupil_to_psf(const float* pupil, const double* kz, const double* z, int64_t nz,
                       int64_t ny, int64_t nx, int normalize, float* psf, void* stream);

/* ---- pupil model (psf/optics.py:96-225, psf/pupil.py:17-97,
 *      psf/aberrations/geometric.py:38-58, psf/aberrations/zernike.py:92-115)
 * FP64 device arrays of ny * nx values (row-major, DC at the corner). */

/* make_geometry: kx, ky (fftfreq grids), kz = sqrt(max(0, (ni/lambda)^2 -
 * kr^2)), rho = kr / (NA/lambda) inside the NA disc else 0, phi = atan2(ky,
 * kx), mask (uint8, kr <= NA/lambda), support (fraction of an oversample x
 * oversample sub-grid inside the disc; oversample 1..32), cos_theta /
 * sin_theta (sin = clip(lambda kr / ni, 0, 1)).  smoothing_sigma > 0 applies
 * the wrapped Gaussian of scipy.ndimage.gaussian_filter (truncate 4, sigma <=
 * 32) to the support, then clips it to [0, 1]; it needs `scratch` (ny * nx
 * doubles).  Errors as the reference: spacing and oversample must be
 * positive, sigma >= 0 (DECON_ERR_VALUE). */
int decon_psf_geometry(int64_t ny, int64_t nx, double dy, double dx, double wavelength, double na,
                       double ni, int oversample, double smoothing_sigma, double* kx, double* ky,
                       double* kz, double* rho, double* phi, uint8_t* mask, double* support,
                       double* cos_theta, double* sin_theta, double* scratch, void* stream);
/* make_pupil: pupil (complex128, interleaved) = support, times the aplanatic
 * factor 1 / sqrt(max(cos theta, eps)) inside the mask when apodize != 0. */
int decon_psf_pupil(const double* support, const double* cos_theta, const uint8_t* mask, int64_t n,
                    int apodize, double* pupil, void* stream);
/* IndexMismatch(depth): pupil *= exp(i 2 pi depth (ns cos t2 - ni cos t1) /
 * lambda), sin t2 = clip((ni / ns) sin t1, 0, 1) (Gibson-Lanni). */
int decon_psf_index_mismatch(const double* sin_theta, const double* cos_theta, int64_t n,
                             double wavelength, double ni, double ns, double depth, double* pupil,
                             void* stream);
/* Defocus(z): pupil *= exp(2 pi i kz z) (psf/aberrations/geometric.py:65-96). */
int decon_psf_defocus(const double* kz, int64_t n, double z, double* pupil, void* stream);
/* ZernikeAberration: pupil *= exp(i mask sum_q coef[q] Z_{j[q]}(rho, phi)),
 * orthonormal OSA/ANSI Zernike polynomials, the sum in the given order (zero
 * coefficients skipped); at most 32 non-zero terms of radial order <= 18.
 * j and coef are host arrays. */
int decon_psf_zernike(const double* rho, const double* phi, const uint8_t* mask, int64_t n,
                      int nterms, const int* j, const double* coef, double* pupil, void* stream);

/* ---- batched RL: many independent problems in one CUDA graph ------------
 * Problem i has its own plan (distinct plans; a plan's scratch spectra serve
 * one problem), observation, background and x / sens / ratio buffers of its
 * plan's signal shape.  The reference solves tiles one at a time
 * (tile_processing.py:226-288); here K iterations of all problems are
 * recorded once into a CUDA graph, forked over `nstreams` internal streams
 * balanced by FFT canvas volume, and replayed.  Pointers are kept, not
 * copied: the buffers must outlive the batch. */
typedef struct decon_batch decon_batch;
int decon_batch_rl_create(int n, decon_conv* const* plans, const float* const* observed,
                          const float* background, float* const* x, float* const* sens,
                          float* const* ratio, int nstreams, decon_batch** out);
/* decon_rl_setup for every problem (x_init may be NULL, or hold NULL entries). */
int decon_batch_rl_setup(decon_batch* b, const float* const* x_init, void* stream);
/* `iterations` iterations of every problem: replays of the cached graph of
 * `iters_per_graph` iterations (captured on first use) plus one remainder
 * graph; ordered after prior work on `stream`, and later work on `stream`
 * waits for it. */
int decon_batch_rl_run(decon_batch* b, int iterations, int iters_per_graph, void* stream);
/* pred_i = A_i x_i + b_i for every problem. */
int decon_batch_rl_predict(decon_batch* b, float* const* pred, void* stream);
/* Kernel nodes in the cached graph of `iters_per_graph` iterations (0 if none). */
int decon_batch_graph_nodes(const decon_batch* b, int iters_per_graph, int64_t* kernels);
int decon_batch_destroy(decon_batch* b);

/* Element-wise RL steps for an arbitrary composed blur operator (the
 * caller runs forward/adjoint through the operator entry points):
 *   decon_rl_ratio:  ratio = y / max(model + b, 1e-10) (rl_mlx.py:147-148);
 *                    ratio may be NULL; if loss_sum != NULL also the FP64
 *                    I-divergence sum (rl_mlx.py:58-80), which needs a
 *                    workspace of decon_reduce_workspace_bytes().
 *   decon_rl_update: x = max(x * (sens>0 ? corr/sens : 0), 1e-10) (:149-150)
 *   decon_rl_data_floor: out = max(y - b, 1e-6) (:123)
 *   decon_rl_mask:   floor = max(max(sens) 1e-6, 1e-10); sens = active ? sens
 *                    : 0; x = active ? max(x, 1e-6) : 0 (:125-133). */
int decon_rl_ratio(const float* model, const float* observed, float background, float* ratio,
                   int64_t n, double* loss_sum, void* workspace, void* stream);
int decon_rl_update(float* x, const float* corr, const float* sens_masked, int64_t n, void* stream);
int decon_rl_data_floor(const float* observed, float background, float* out, int64_t n, void* stream);
int decon_rl_mask(float* x, float* sens, int64_t n, void* workspace, void* stream);
int decon_fill(float* p, float value, int64_t n, void* stream);
int decon_clamp_min(const float* a, float lo, float* out, int64_t n, void* stream);
/* out = alpha a + beta (pred = A x + b, rl_mlx.py:174). */
int decon_affine(const float* a, float alpha, float beta, float* out, int64_t n, void* stream);

/* ---- adaptive PDHG (deconvolution/pdhg_mlx.py:507-1242) ------------------ */

typedef struct decon_pdhg decon_pdhg; /* device-resident tau/sigma/theta + histories */

/* State for one solve: tau = sigma = step_scale, theta = 1 (pdhg_mlx.py:693-701).
 * Every kernel below reads the step sizes from this state and returns at
 * once after the stop flag is set (convergence or num_iter reached), so a
 * host can queue iterations without synchronising. */
int decon_pdhg_create(int num_iter, double step_scale, double delta, double eta, double tol,
                      int min_iter, int patience, decon_pdhg** out);
/* Start a new solve in an existing state (same meaning as decon_pdhg_create;
 * num_iter must not exceed the num_iter the state was created with).  Queued
 * on `stream`; no allocation, so pooled states cost no cudaFree.  The
 * reference creates fresh scalars per call (pdhg_mlx.py:693-701). */
int decon_pdhg_reset(decon_pdhg* h, int num_iter, double step_scale, double delta, double eta,
                     double tol, int min_iter, int patience, void* stream);
int decon_pdhg_destroy(decon_pdhg* h);
/* y1 = prox_{sigma F*}(y1 + sigma ((1+theta) Ax_cur - theta Ax_prev)),
 * loss_type 0 Poisson (pdhg_mlx.py:115-166), 1 Gaussian (:169-189). */
int decon_pdhg_dual_data(decon_pdhg* h, float* y1, const float* ax_cur, const float* ax_prev,
                         const float* data, float background, int loss_type, int64_t m,
                         void* stream);
/* y2 = proj(y2 + sigma L xbar); norm 0 L1 clip, 1 L1,2 ball (pdhg_mlx.py:197-233).
 * y2, lxbar: (ncomp, n). */
int decon_pdhg_dual_reg(decon_pdhg* h, float* y2, const float* lxbar, float alpha, int norm,
                        int ncomp, int64_t n, void* stream);
/* xbar = x_cur + theta (x_cur - x_prev) (pdhg_mlx.py:841). */
int decon_pdhg_xbar(decon_pdhg* h, const float* xc, const float* xp, float* xbar, int64_t n,
                    void* stream);
/* x_new = max(0, x - tau (aty + lty)) plus FP64 ||dx||^2, ||x||^2, ||x_new||^2
 * (pdhg_mlx.py:741-750, 805-806); lty may be NULL. */
int decon_pdhg_primal(decon_pdhg* h, const float* xc, const float* aty, const float* lty,
                      float* xn, int64_t n, void* stream);
int decon_pdhg_sub(decon_pdhg* h, const float* a, const float* b, float* d, int64_t n, void* stream);
/* ||A x_new - A x||^2 and (l_dx != NULL) ||L (x_new - x)||^2 (pdhg_mlx.py:753-759). */
int decon_pdhg_dk(decon_pdhg* h, const float* ax_new, const float* ax_cur, int64_t m,
                  const float* l_dx, int64_t nl, void* stream);
/* Malitsky-Pock step-size update and convergence test in FP64 (pdhg_mlx.py:761-857). */
int decon_pdhg_step(decon_pdhg* h, void* stream);
/* Objective at iteration k (pdhg_mlx.py:860-881): data term of (ax + b, data)
 * plus alpha times the L1 / L1,2 norm of lx (ncomp, n). */
int decon_pdhg_loss(decon_pdhg* h, const float* ax, const float* data, float background,
                    int loss_type, int64_t m, const float* lx, int norm, int ncomp, int64_t n,
                    double alpha, int k, void* stream);
/* Fused Hessian3D forms of the regulariser half (L = Hessian3D(r), shape
 * (z, y, x)); the Hessian is evaluated on the fly, never stored:
 *   hess_dual:   y2 = proj(y2 + sigma H x_bar), x_bar = x + theta (x - x_prev)
 *   hess_primal: x_new = max(0, x - tau (aty + H^T y2)) + the FP64 sums of
 *                decon_pdhg_primal
 *   hess_dk:     ||A x_new - A x||^2 and ||H (x_new - x)||^2 (ax_new NULL:
 *                only the Hessian term, so that it may run beside the
 *                forward convolution; decon_pdhg_dk(l_dx = NULL) adds the
 *                data term)
 *   hess_loss:   objective at iteration k with the H x_new norm fused. */
int decon_pdhg_hess_dual(decon_pdhg* h, float* y2, const float* xc, const float* xp,
                         const int64_t shape[3], float r, float alpha, int norm, void* stream);
int decon_pdhg_hess_primal(decon_pdhg* h, const float* xc, const float* aty, const float* y2,
                           float* xn, const int64_t shape[3], float r, void* stream);
/* hess_dual followed by hess_primal in one kernel (pdhg_mlx.py:732-743):
 * y2_out = proj(y2_in + sigma H x_bar), then x_new = max(0, x - tau (aty +
 * H^T y2_out)) and its FP64 sums, with y2_out consumed from shared memory
 * (each tile recomputes the y2_out values of its one-voxel halo).  y2_in and
 * y2_out are distinct buffers (6, z, y, x): alternate them between
 * iterations.  Same float32 values as the two separate calls. */
int decon_pdhg_hess_dual_primal(decon_pdhg* h, const float* y2_in, float* y2_out, const float* xc,
                                const float* xp, const float* aty, float* xn,
                                const int64_t shape[3], float r, float alpha, int norm,
                                void* stream);
int decon_pdhg_hess_dk(decon_pdhg* h, const float* ax_new, const float* ax_cur, int64_t m,
                       const float* xn, const float* xc, const int64_t shape[3], float r,
                       void* stream);
int decon_pdhg_hess_loss(decon_pdhg* h, const float* ax, const float* data, float background,
                         int loss_type, int64_t m, const float* x, const int64_t shape[3], float r,
                         int norm, double alpha, int k, void* stream);
/* Reads the state (synchronises): iteration counter, final iteration,
 * converged and stop flags, (tau, sigma, theta) and the histories (host
 * arrays of num_iter doubles; any may be NULL). */
int decon_pdhg_read(decon_pdhg* h, int* k, int* final_iter, int* converged, int* stop,
                    double* scalars3, double* tau_hist, double* sigma_hist, double* loss_hist,
                    double* rel_hist, void* stream);
/* Host-requested stop (a callback returned truthy). Synchronises. */
int decon_pdhg_set_stop(decon_pdhg* h, int final_iter, void* stream);
/* Queues a copy of {k, count, converged, final_iter, stop} (5 int32) into
 * host_status (page-locked host memory for the copy to stay asynchronous);
 * the values are valid once the stream has passed this point.  Lets a host
 * that drives many solves poll convergence without synchronising (no
 * reference counterpart: the reference reads float(rel_change) every
 * iteration, pdhg_mlx.py:810). */
int decon_pdhg_status_async(decon_pdhg* h, int32_t* host_status, void* stream);

/* ---- resident Hessian-PDHG solve (pdhg_mlx.py:507-900) ------------------ */

typedef struct decon_pdhg_solver decon_pdhg_solver; /* x, A x, duals, tables */

/* solve_pdhg_mlx with regularization="hessian" (pdhg_mlx.py:507-700 set-up)
 * as one device-resident object: A = FractionalAreaDownsample(scale) o
 * LinearFFTConvolver(conv) (conv's signal shape N is the object shape;
 * data_shape M the observation's, M[a] == N[a] on axes that are not
 * resampled; all scale[a] == 1 is the plain operator A = conv), Hessian3D
 * with spacing ratio r, norm 0 = L1 / 1 = L1_2, loss 0 = Poisson / 1 =
 * Gaussian.  data: device, shape M (copied).  x0: device, shape N, clamped
 * at 0; NULL = the reference's default (max(A^T data, 0) when resampled,
 * max(data, 0) for the plain operator).  The plan `conv` must outlive the
 * solver.  Allocates its buffers (x and A x twice, y1, six-component y2,
 * A^T y1, two resampling intermediates); queues the initial state on
 * `stream`. */
int decon_pdhg_solver_create(decon_conv* conv, const float* data, const int64_t data_shape[3],
                             const double scale[3], float background, int loss_type,
                             const float* x0, double r, double alpha, int norm, int num_iter,
                             double delta, double eta, double tol, int min_iter, int patience,
                             int eval_interval, void* stream, decon_pdhg_solver** out);
/* Queues up to `iterations` more iterations of the PDHG loop
 * (pdhg_mlx.py:717-900; at most num_iter in total), each the fused launch
 * sequence dual / A^T / Hessian dual / primal / A / ||dK x||^2 / FP64 step,
 * plus the loss every eval_interval iterations.  No host synchronisation and
 * no allocation: the calls may be captured in a CUDA graph.  Iterations
 * after convergence are no-ops on the device. */
int decon_pdhg_run(decon_pdhg_solver* s, int iterations, void* stream);
/* Copies x of the last completed iteration (the converged iterate if the
 * solve stopped early) to x_out (device, shape N).  Synchronises. */
int decon_pdhg_solver_x(decon_pdhg_solver* s, float* x_out, void* stream);
/* The solver's scalar state (read it with decon_pdhg_read) and the number of
 * iterations queued so far. */
int decon_pdhg_solver_state(decon_pdhg_solver* s, decon_pdhg** state, int* queued);
int decon_pdhg_solver_destroy(decon_pdhg_solver* s);

/* ---- pad / crop (deconvolution/core_operators.py:29-137) ---------------- */

/* Copies the box [start, start + ext) of src (shape src_shape) to dst at
 * dst_start inside dst_shape; every other dst element is set to zero.  One
 * kernel serves Pad.forward/adjoint and Crop.forward/adjoint. ndim <= 4. */
int decon_window_copy(const float* src, const int64_t* src_shape, const int64_t* src_start,
                      float* dst, const int64_t* dst_shape, const int64_t* dst_start,
                      const int64_t* ext, int ndim, void* stream);

/* ---- fractional-area resampling (core_operators.py:151-450) ------------- */

/* Band tables of _banded_overlap_weights_1d (core_operators.py:151-202),
 * computed on the host in FP64 and rounded to float32.  widths via
 * decon_band_widths.  Host arrays. */
int decon_band_widths(int64_t n_large, int64_t n_small, int* w_fwd, int* w_adj);
int decon_band_weights(int64_t n_large, int64_t n_small, int32_t* idx_fwd, float* w_fwd,
                       int32_t* idx_adj, float* w_adj);
/* out[o, i, q] = sum_k w[i,k] * in[o, idx[i,k], q] along one axis
 * (_apply_banded_1d, core_operators.py:205-219).  in: (outer, n_in, inner),
 * out: (outer, n_out, inner); idx/w: device (n_out, width). */
int decon_banded_axis(const float* in, float* out, int64_t outer, int64_t n_in, int64_t inner,
                      int64_t n_out, const int32_t* idx, const float* w, int width, void* stream);

/* ---- finite-difference operators (linops_mlx.py:92-262) ----------------- */

/* Hessian3D.forward: h[6, z, y, x] = [r^2 zz, yy, xx, sqrt2 r yz, sqrt2 r xz,
 * sqrt2 xy] with Neumann boundaries (linops_mlx.py:224-242). */
int decon_hessian3d_forward(const float* x, float* h, const int64_t shape[3], float r,
                            void* stream);
/* Hessian3D.adjoint (linops_mlx.py:244-259). */
int decon_hessian3d_adjoint(const float* h, float* x, const int64_t shape[3], float r,
                            void* stream);
/* Gradient3D.forward / adjoint (linops_mlx.py:107-119). */
int decon_gradient3d_forward(const float* x, float* g, const int64_t shape[3], float r,
                             void* stream);
int decon_gradient3d_adjoint(const float* g, float* x, const int64_t shape[3], float r,
                             void* stream);

/* ---- reductions (FP64, deterministic) ----------------------------------- */

#define DECON_RED_SUM 0      /* sum a                          */
#define DECON_RED_SUMSQ 1    /* sum a^2                        */
#define DECON_RED_DIFFSQ 2   /* sum (a - b)^2                  */
#define DECON_RED_MAX 3      /* max a                          */
#define DECON_RED_DOT 4      /* sum a b                        */
/* Bytes of device workspace decon_reduce needs (per concurrent call). */
int64_t decon_reduce_workspace_bytes(void);
/* out[0] (device double) = reduction over n elements of a (and b).  Two
 * fixed-shape passes, so the result is bitwise reproducible run to run.
 * workspace: caller-owned device buffer of decon_reduce_workspace_bytes();
 * calls that share a workspace must be ordered on one stream.  This is the
 * FP64 reduction the solvers use for norms, flux and step sizes
 * (pdhg_mlx.py:750,759,805-809; rl_mlx.py:77-80,130). */
int decon_reduce(const float* a, const float* b, int64_t n, int op, double* out, void* workspace,
                 void* stream);

/* The reduction above for callers that cannot allocate device memory (no
 * counterpart in the reference): plug-ins inside a host application that owns
 * every device allocation, or pipelines that reserve memory up front because
 * cudaMalloc can synchronise the device and fail at run time.  It allocates
 * nothing: its scratch is a fixed 128 KB device array inside the library
 * (held by every GPU that loads it until exit), so n is limited to
 * 67,108,864 elements (DECON_ERR_VALUE beyond).  The first call on a device
 * looks up that array's address with the device current, and looks it up
 * again after the device's context changed (cudaDeviceReset); make that
 * first call before any stream capture.  All calls share the array: calls
 * whose kernels overlap on the GPU race, so order them on one stream. */
int decon_reduce_noalloc(const float* a, const float* b, int64_t n, int op, double* out,
                         void* stream);

/* ---- kernel timing (no reference counterpart: measurement support) ------ */

#define DECON_PROF_XR2C 1 /* X R2C pass              */
#define DECON_PROF_COL 2  /* Y / inverse-Y passes    */
#define DECON_PROF_ZOTF 4 /* axial FFT x OTF x IFFT  */
#define DECON_PROF_XC2R 8 /* X C2R pass + epilogue   */
/* Records CUDA events on the launching stream around every launch of the
 * selected FFT pass classes until decon_profile_stop, which synchronises,
 * returns the summed kernel time (ms) and launch count, and disables timing.
 * Process-wide, not thread-safe; for benchmarks. */
int decon_profile_start(int class_mask);
int decon_profile_stop(double* ms_total, int64_t* launches);

#ifdef __cplusplus
}
#endif

#endif /* DECON_B200_H */
