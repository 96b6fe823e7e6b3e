"""B200-native (sm_100a) non-rigid warp-field solve behind CUDAFusion's
GaussNewtonSolver / WarpField call surface."""
__version__ = "0.1.0"
