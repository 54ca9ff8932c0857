// decon_pdhg_run: N resident Hessian-PDHG iterations behind one C call.
//
// The solver object holds everything solve_pdhg_mlx's loop keeps between
// iterations (deconlib/deconvolution/pdhg_mlx.py:717-900) on the device:
// x triple-buffered (slot k % 3 holds iteration k's, slot (k + 2) % 3 the
// previous one's, x_new goes to slot (k + 1) % 3), A x double-buffered (slot
// k % 2), the duals y1 (data) and y2 (six Hessian components, double-buffered:
// slot k % 2 is read, the other written), A^T y1, the intermediate volumes of
// the resampling passes and their band tables.  One iteration is the launch
// sequence of the fused Hessian path:
//
//   y1   = prox(y1 + sigma A x_bar)        A x_bar from the two A x slots
//   A^T y1                                  banded adjoint passes, conv adjoint
//   y2'  = proj(y2 + sigma H x_bar)        Hessian dual kernel
//   x_new = max(0, x - tau (A^T y1 + H^T y2')) + FP64 sums
//                                           Hessian primal kernel (or both in
//                                           one z-walk, DECON_FUSED_STENCIL=1)
//   A x_new                                 conv forward, banded passes
//   ||A dx||^2, ||H dx||^2                  FP64 sums
//   Malitsky-Pock step (FP64, one CTA), loss every eval_interval iterations
//
// Nothing here reads a device scalar back or allocates after creation, so a
// caller may queue any number of iterations (or capture them in a CUDA
// graph); a converged or finished solve turns the remaining iterations into
// no-ops on the device.
#include <cmath>
#include <cstdlib>
#include <vector>

#include "conv_impl.cuh"
#include "solvers.cuh"

struct decon_pdhg_solver {
    decon_conv* conv = nullptr;
    decon_pdhg* state = nullptr;
    int64_t N[3] = {1, 1, 1}, M[3] = {1, 1, 1};
    int64_t n = 0, m = 0;
    float bg = 0.f, r = 1.f, alpha = 0.f;  // float32 copies the kernels take
    double alpha_d = 0.0;                  // the loss weight in FP64
    int loss = 0, norm = 0, eval_interval = 10, num_iter = 0;
    int k = 0;  // iterations queued so far
    // device buffers
    float* X[3] = {nullptr, nullptr, nullptr};
    float* AX[2] = {nullptr, nullptr};
    float* Y2[2] = {nullptr, nullptr};
    float *y1 = nullptr, *aty = nullptr, *data = nullptr;
    float *t0 = nullptr, *t1 = nullptr;  // resampling intermediates
    // resampling passes in application order of the forward operator
    struct Band {
        int axis;
        int64_t nl, ns;
        int wf, wa;
        int32_t *idx_f, *idx_a;
        float *w_f, *w_a;
    };
    std::vector<Band> bands;
    // every axis halved exactly: A and A^T as the fused 2x area-sum passes
    bool down2 = false;
    // dual + primal Hessian updates in one z-walk (DECON_FUSED_STENCIL=1 at
    // creation) or as two kernels (default: measured faster on the B200)
    bool fused_stencil = false;
    std::vector<void*> allocs;
};

namespace dk {

static int pr_alloc(decon_pdhg_solver* s, void** p, size_t bytes) {
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    const cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(DECON_ERR_OOM, "decon_pdhg_solver: cudaMalloc of %zu bytes failed: %s", bytes,
                    cudaGetErrorString(e));
    }
    s->allocs.push_back(*p);
    return DECON_OK;
}

// One banded pass along `axis` of a volume of shape `shp` (updated to the
// output shape).
static int pr_band(const decon_pdhg_solver::Band& b, bool adjoint, const float* in, float* out,
                   int64_t shp[3], cudaStream_t st) {
    const int a = b.axis;
    int64_t outer = 1, inner = 1;
    for (int i = 0; i < a; ++i) outer *= shp[i];
    for (int i = a + 1; i < 3; ++i) inner *= shp[i];
    const int64_t n_in = shp[a], n_out = adjoint ? b.nl : b.ns;
    DK_TRY(decon_banded_axis(in, out, outer, n_in, inner, n_out, adjoint ? b.idx_a : b.idx_f,
                             adjoint ? b.w_a : b.w_f, adjoint ? b.wa : b.wf, st));
    shp[a] = n_out;
    return DECON_OK;
}

// A x (N-space x -> M-space out): convolution, then the banded passes in
// axis order (FractionalAreaDownsample.forward, core_operators.py:301-320).
static int pr_forward(decon_pdhg_solver* s, const float* x, float* out, cudaStream_t st) {
    if (s->bands.empty()) return decon_conv_forward(s->conv, x, out, st);
    if (s->down2) {
        const int e = decon_conv_forward_down2(s->conv, x, out, st);
        if (e != DECON_ERR_UNSUPPORTED) return e;
        s->down2 = false;
    }
    DK_TRY(decon_conv_forward(s->conv, x, s->t0, st));
    int64_t shp[3] = {s->N[0], s->N[1], s->N[2]};
    const float* cur = s->t0;
    for (size_t i = 0; i < s->bands.size(); ++i) {
        float* dst = i + 1 == s->bands.size() ? out : (cur == s->t0 ? s->t1 : s->t0);
        DK_TRY(pr_band(s->bands[i], false, cur, dst, shp, st));
        cur = dst;
    }
    return DECON_OK;
}

// A^T y (M-space y -> N-space out): the banded adjoint passes in axis order
// (core_operators.py:322-336), then the convolution adjoint.
static int pr_adjoint(decon_pdhg_solver* s, const float* y, float* out, cudaStream_t st) {
    if (s->bands.empty()) return decon_conv_adjoint(s->conv, y, out, st);
    if (s->down2) {
        const int e = decon_conv_adjoint_up2(s->conv, y, out, st);
        if (e != DECON_ERR_UNSUPPORTED) return e;
        s->down2 = false;
    }
    int64_t shp[3] = {s->M[0], s->M[1], s->M[2]};
    const float* cur = y;
    for (size_t i = 0; i < s->bands.size(); ++i) {
        float* dst = cur == s->t0 ? s->t1 : s->t0;
        DK_TRY(pr_band(s->bands[i], true, cur, dst, shp, st));
        cur = dst;
    }
    return decon_conv_adjoint(s->conv, cur, out, st);
}

}  // namespace dk

extern "C" {

int decon_pdhg_solver_create(decon_conv* conv, const float* data, const int64_t data_shape[3],
                             const double scale[3], float background, int loss_type,
                             const float* x0, double r, double alpha, int norm, int num_iter,
                             double delta, double eta, double tol, int min_iter, int patience,
                             int eval_interval, void* stream, decon_pdhg_solver** out) {
    using namespace dk;
    if (!conv || !data || !data_shape || !scale || !out) return fail(DECON_ERR_NULL, "null pointer");
    *out = nullptr;
    if (loss_type != 0 && loss_type != 1) return fail(DECON_ERR_VALUE, "loss_type must be 0 or 1");
    if (norm != 0 && norm != 1) return fail(DECON_ERR_VALUE, "norm must be 0 (L1) or 1 (L1_2)");
    if (num_iter < 0) return fail(DECON_ERR_VALUE, "num_iter must be >= 0");
    if (eval_interval < 1) return fail(DECON_ERR_VALUE, "eval_interval must be >= 1");
    const cudaStream_t st = as_stream(stream);
    decon_pdhg_solver* s = new (std::nothrow) decon_pdhg_solver();
    if (!s) return fail(DECON_ERR_OOM, "host allocation failed");
    auto bail = [&](int code) {
        decon_pdhg_solver_destroy(s);
        return code;
    };
    for (int i = 0; i < 3; ++i) {
        s->N[i] = conv->N[i];
        s->M[i] = data_shape[i];
        if (s->M[i] < 1 || s->M[i] > s->N[i] || !(scale[i] >= 1.0))
            return bail(fail(DECON_ERR_VALUE,
                             "decon_pdhg_solver_create: axis %d: data extent %lld must lie in "
                             "[1, %lld] and scale %g must be >= 1",
                             i, (long long)s->M[i], (long long)s->N[i], scale[i]));
    }
    s->conv = conv;
    s->n = s->N[0] * s->N[1] * s->N[2];
    s->m = s->M[0] * s->M[1] * s->M[2];
    s->bg = background;
    s->r = (float)r;
    s->alpha = (float)alpha;
    s->alpha_d = alpha;
    s->loss = loss_type;
    s->norm = norm;
    s->eval_interval = eval_interval;
    s->num_iter = num_iter;
    double down_norm = 1.0;
    bool plain = true;
    for (int a = 0; a < 3; ++a) {
        down_norm *= scale[a];
        if (scale[a] != 1.0) plain = false;
        if (s->N[a] == s->M[a]) continue;
        decon_pdhg_solver::Band b{};
        b.axis = a;
        b.nl = s->N[a];
        b.ns = s->M[a];
        if (int e = decon_band_widths(b.nl, b.ns, &b.wf, &b.wa)) return bail(e);
        std::vector<int32_t> i_f((size_t)b.ns * b.wf), i_a((size_t)b.nl * b.wa);
        std::vector<float> w_f(i_f.size()), w_a(i_a.size());
        if (int e = decon_band_weights(b.nl, b.ns, i_f.data(), w_f.data(), i_a.data(), w_a.data()))
            return bail(e);
        void* p = nullptr;
        if (int e = pr_alloc(s, &p, i_f.size() * 4)) return bail(e);
        b.idx_f = (int32_t*)p;
        if (int e = pr_alloc(s, &p, i_a.size() * 4)) return bail(e);
        b.idx_a = (int32_t*)p;
        if (int e = pr_alloc(s, &p, w_f.size() * 4)) return bail(e);
        b.w_f = (float*)p;
        if (int e = pr_alloc(s, &p, w_a.size() * 4)) return bail(e);
        b.w_a = (float*)p;
        if (int e = upload_blocking(b.idx_f, i_f.data(), i_f.size() * 4)) return bail(e);
        if (int e = upload_blocking(b.idx_a, i_a.data(), i_a.size() * 4)) return bail(e);
        if (int e = upload_blocking(b.w_f, w_f.data(), w_f.size() * 4)) return bail(e);
        if (int e = upload_blocking(b.w_a, w_a.data(), w_a.size() * 4)) return bail(e);
        s->bands.push_back(b);
    }
    s->down2 = s->bands.size() == 3;
    for (const auto& b : s->bands) s->down2 = s->down2 && b.nl == 2 * b.ns;
    if (s->bands.empty() && (s->M[0] != s->N[0] || s->M[1] != s->N[1] || s->M[2] != s->N[2]))
        return bail(fail(DECON_ERR_VALUE, "decon_pdhg_solver_create: shape mismatch"));
    // buffers
    void* p = nullptr;
    for (int i = 0; i < 3; ++i) {
        if (int e = pr_alloc(s, &p, (size_t)s->n * 4)) return bail(e);
        s->X[i] = (float*)p;
    }
    s->fused_stencil = getenv("DECON_FUSED_STENCIL") != nullptr;
    for (int i = 0; i < 2; ++i) {
        if (int e = pr_alloc(s, &p, (size_t)s->m * 4)) return bail(e);
        s->AX[i] = (float*)p;
        if (i == 1 && !s->fused_stencil) continue;  // the two-kernel form updates y2 in place
        if (int e = pr_alloc(s, &p, (size_t)6 * s->n * 4)) return bail(e);
        s->Y2[i] = (float*)p;
    }
    if (int e = pr_alloc(s, &p, (size_t)s->m * 4)) return bail(e);
    s->y1 = (float*)p;
    if (int e = pr_alloc(s, &p, (size_t)s->m * 4)) return bail(e);
    s->data = (float*)p;
    if (int e = pr_alloc(s, &p, (size_t)s->n * 4)) return bail(e);
    s->aty = (float*)p;
    if (!s->bands.empty()) {
        // the largest intermediate of the axis passes is at most N voxels
        if (int e = pr_alloc(s, &p, (size_t)s->n * 4)) return bail(e);
        s->t0 = (float*)p;
        if (int e = pr_alloc(s, &p, (size_t)s->n * 4)) return bail(e);
        s->t1 = (float*)p;
    }
    // state: step_scale = 0.99 / sqrt(||A||^2 + ||H||^2) (pdhg_mlx.py:697-700)
    const double a_norm = plain ? conv->norm_sq : down_norm * conv->norm_sq;
    const double rr = r;
    const double h_norm = 16.0 * rr * rr * rr * rr + 4.0 * rr * rr + 34.0;
    const double step_scale = 0.99 / std::sqrt(a_norm + h_norm);
    if (int e = decon_pdhg_create(num_iter, step_scale, delta, eta, tol, min_iter, patience, &s->state))
        return bail(e);
    // initial state on the caller's stream: data copy, x0, A x0, zero duals
    if (cudaMemcpyAsync(s->data, data, (size_t)s->m * 4, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return bail(fail(DECON_ERR_CUDA, "copy of the observation failed"));
    if (x0) {
        if (int e = decon_clamp_min(x0, 0.f, s->X[0], s->n, st)) return bail(e);
    } else if (plain) {
        if (int e = decon_clamp_min(s->data, 0.f, s->X[0], s->n, st)) return bail(e);
    } else {
        if (int e = pr_adjoint(s, s->data, s->aty, st)) return bail(e);
        if (int e = decon_clamp_min(s->aty, 0.f, s->X[0], s->n, st)) return bail(e);
    }
    for (int i = 1; i < 3; ++i)
        if (cudaMemcpyAsync(s->X[i], s->X[0], (size_t)s->n * 4, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
            return bail(fail(DECON_ERR_CUDA, "copy of x0 failed"));
    if (int e = pr_forward(s, s->X[0], s->AX[0], st)) return bail(e);
    if (cudaMemcpyAsync(s->AX[1], s->AX[0], (size_t)s->m * 4, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return bail(fail(DECON_ERR_CUDA, "copy of A x0 failed"));
    if (cudaMemsetAsync(s->y1, 0, (size_t)s->m * 4, st) != cudaSuccess ||
        cudaMemsetAsync(s->Y2[0], 0, (size_t)6 * s->n * 4, st) != cudaSuccess)
        return bail(fail(DECON_ERR_CUDA, "clearing the duals failed"));
    *out = s;
    return DECON_OK;
}

int decon_pdhg_run(decon_pdhg_solver* s, int iterations, void* stream) {
    using namespace dk;
    if (!s) return fail(DECON_ERR_NULL, "null pointer");
    if (iterations < 0) return fail(DECON_ERR_VALUE, "iterations must be >= 0");
    const cudaStream_t st = as_stream(stream);
    decon_pdhg* h = s->state;
    const int64_t* shp = s->N;
    for (int it = 0; it < iterations && s->k < s->num_iter; ++it) {
        const int k = s->k;
        float* xc = s->X[k % 3];
        float* xp = s->X[(k + 2) % 3];
        float* xn = s->X[(k + 1) % 3];
        float* axc = s->AX[k % 2];
        float* axn = s->AX[(k + 1) % 2];  // holds A x_{k-1}; overwritten with A x_new
        DK_TRY(decon_pdhg_dual_data(h, s->y1, axc, axn, s->data, s->bg, s->loss, s->m, st));
        DK_TRY(pr_adjoint(s, s->y1, s->aty, st));
        if (s->fused_stencil) {
            DK_TRY(decon_pdhg_hess_dual_primal(h, s->Y2[k % 2], s->Y2[(k + 1) % 2], xc, xp, s->aty,
                                               xn, shp, s->r, s->alpha, s->norm, st));
        } else {
            // y2 updated in place in slot 0
            DK_TRY(decon_pdhg_hess_dual(h, s->Y2[0], xc, xp, shp, s->r, s->alpha, s->norm, st));
            DK_TRY(decon_pdhg_hess_primal(h, xc, s->aty, s->Y2[0], xn, shp, s->r, st));
        }
        DK_TRY(pr_forward(s, xn, axn, st));
        // ||A dx||^2 and ||H dx||^2 as two sums (the split the two-stream
        // Python driver uses, so both drivers give the same bits)
        DK_TRY(decon_pdhg_dk(h, axn, axc, s->m, nullptr, 0, st));
        DK_TRY(decon_pdhg_hess_dk(h, nullptr, nullptr, 0, xn, xc, shp, s->r, st));
        DK_TRY(decon_pdhg_step(h, st));
        if ((k + 1) % s->eval_interval == 0)
            DK_TRY(decon_pdhg_hess_loss(h, axn, s->data, s->bg, s->loss, s->m, xn, shp, s->r,
                                        s->norm, s->alpha_d, k, st));
        s->k = k + 1;
    }
    return DECON_OK;
}

int decon_pdhg_solver_x(decon_pdhg_solver* s, float* x_out, void* stream) {
    using namespace dk;
    if (!s || !x_out) return fail(DECON_ERR_NULL, "null pointer");
    int k = 0, final_iter = 0;
    DK_TRY(decon_pdhg_read(s->state, &k, &final_iter, nullptr, nullptr, nullptr, nullptr, nullptr,
                           nullptr, nullptr, stream));
    const int fi = s->num_iter > 0 ? std::min(final_iter, s->k) : 0;
    DK_CUDA(cudaMemcpyAsync(x_out, s->X[fi % 3], (size_t)s->n * 4, cudaMemcpyDeviceToDevice,
                            as_stream(stream)));
    return DECON_OK;
}

int decon_pdhg_solver_state(decon_pdhg_solver* s, decon_pdhg** state, int* queued) {
    using namespace dk;
    if (!s || !state) return fail(DECON_ERR_NULL, "null pointer");
    *state = s->state;
    if (queued) *queued = s->k;
    return DECON_OK;
}

int decon_pdhg_solver_destroy(decon_pdhg_solver* s) {
    if (!s) return DECON_OK;
    if (s->state) decon_pdhg_destroy(s->state);
    for (void* p : s->allocs) cudaFree(p);
    delete s;
    return DECON_OK;
}

}  // extern "C"
