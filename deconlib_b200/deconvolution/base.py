"""Result record of the PDHG solvers (deconvolution/base.py:15-34 in deconlib)."""

from dataclasses import dataclass, field
from typing import Any, List

__all__ = ["MLXDeconvolutionResult"]


@dataclass
class MLXDeconvolutionResult:
    """restored (CUDA tensor), iterations, loss/tau/sigma histories, converged, metadata."""

    restored: Any
    iterations: int
    loss_history: List[float] = field(default_factory=list)
    converged: bool = False
    tau_history: List[float] = field(default_factory=list)
    sigma_history: List[float] = field(default_factory=list)
    metadata: dict = field(default_factory=dict)
