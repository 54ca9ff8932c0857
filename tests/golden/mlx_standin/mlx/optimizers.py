"""Empty stand-in for mlx.optimizers; the deconvolution path never calls it."""
