"""Empty stand-in for h5py: deconlib imports it at package load; the deconvolution path never calls it."""
