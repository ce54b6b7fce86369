"""augurv2_b200 - B200 (sm_100a) backend for the MCMC samplers that AugurV2
compiles: hand-written CUDA for the data-parallel hot path behind the
reference's AugurInfer API (augurv2_b200.augurlib)."""
__version__ = "0.1.0"
