// Device-resident PDHG state shared by the solver kernels.
#pragma once

#include "common.cuh"

namespace dk {

constexpr int kPdhgGrid = 592;   // fixed grid of the reducing kernels (4 per SM)
constexpr int kPdhgSlots = 8;    // FP64 partial-sum slots

struct PdhgDev {
    double tau, sigma, theta;
    double step_scale, delta, eta, tol;
    double last_dx2, last_dK2;
    int k, count, converged, final_iter, stop, min_iter, patience, num_iter;
    double* tau_hist;
    double* sigma_hist;
    double* loss_hist;
    double* rel_hist;
    double* partials;  // [kPdhgSlots][kPdhgGrid]
};

}  // namespace dk

struct decon_pdhg {
    void* mem = nullptr;
    dk::PdhgDev* dev = nullptr;
    int num_iter = 0;
    int capacity = 0;  // history length allocated (decon_pdhg_reset accepts num_iter <= capacity)
};
