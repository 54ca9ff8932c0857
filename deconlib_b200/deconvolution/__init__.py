"""Drop-in B200 implementation of deconlib's deconvolution hot path.

Same names and signatures as ``deconlib.deconvolution`` for the operator
algebra (LinearFFTConvolver, FFTConvolver, Pad, Crop,
FractionalAreaDownsample / Upsample, Hessian / Gradient, compose) and the
solvers (richardson_lucy_with_operator, solve_pdhg_mlx,
solve_pdhg_with_operator, nlcg_with_operator).  Arrays are CUDA
``torch.Tensor`` float32; NumPy input is copied to the device.
"""

from .base import MLXDeconvolutionResult
from .composition import Compose, LinearOperator, as_numpy_op, compose
from .core_operators import Crop, FractionalAreaDownsample, FractionalAreaUpsample, Pad
from .linops import (FFTConvolver, Gradient1D, Gradient2D, Gradient3D, Hessian1D, Hessian2D,
                     Hessian3D, LinearFFTConvolver, STATIC_FFT_LENGTHS, fast_padded_shape,
                     pad_corner_origin_kernel, static_fft_shape)
from .pdhg import (GradientRegularizer, HessianRegularizer, IdentityRegularizer, PDHGRunner,
                   pdhg_mlx_runner, pdhg_result, prox_gaussian_dual, prox_l1_2_dual, prox_l1_dual,
                   prox_nonneg, prox_poisson_dual, solve_pdhg_mlx, solve_pdhg_with_operator)
from .nlcg import (NLCGResult, i_divergence_between, nlcg_gradient, nlcg_hessian_quadform,
                   nlcg_objective, nlcg_solver, nlcg_step_length, nlcg_with_operator)
from .rl import (RLResult, RLRunner, poisson_i_divergence, richardson_lucy_solver,
                 richardson_lucy_with_operator)
from .shapes import compute_padded_shape, compute_visible_shape, get_valid_slices
from .forward_model import ForwardModel, make_forward_model
from .tile_processing import TilePlan, TileSpec, optimal_tile_size, plan_tiles, process_tiles

__all__ = [
    "MLXDeconvolutionResult", "Compose", "LinearOperator", "as_numpy_op", "compose", "Crop",
    "FractionalAreaDownsample", "FractionalAreaUpsample", "Pad", "FFTConvolver", "Gradient1D",
    "Gradient2D", "Gradient3D", "Hessian1D", "Hessian2D", "Hessian3D", "LinearFFTConvolver",
    "fast_padded_shape", "static_fft_shape", "STATIC_FFT_LENGTHS", "pad_corner_origin_kernel",
    "GradientRegularizer", "HessianRegularizer",
    "IdentityRegularizer", "prox_gaussian_dual", "prox_l1_2_dual", "prox_l1_dual", "prox_nonneg",
    "prox_poisson_dual", "solve_pdhg_mlx", "solve_pdhg_with_operator", "RLResult",
    "poisson_i_divergence", "richardson_lucy_solver", "richardson_lucy_with_operator",
    "RLRunner", "PDHGRunner", "pdhg_mlx_runner", "pdhg_result", "compute_padded_shape",
    "compute_visible_shape", "get_valid_slices", "ForwardModel", "make_forward_model", "TilePlan",
    "TileSpec", "optimal_tile_size", "plan_tiles", "process_tiles", "NLCGResult",
    "nlcg_with_operator", "nlcg_solver", "nlcg_objective", "nlcg_gradient",
    "nlcg_hessian_quadform", "nlcg_step_length", "i_divergence_between",
]
