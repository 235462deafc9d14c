"""Seeded synthetic GP problems (stand-ins for the reference's time-series
dataset, which is not available): inputs X ~ U[0,1]^(N x d) and targets
y = sin(sum_k x_ik) + N(0, noise_sd^2), drawn with numpy's PCG64."""
import numpy as np

# name -> N, d, lengthscale, sf2, sn2, matrixBlockSize, CG epsilon
CONFIGS = {
    "c1_n4096": dict(N=4096, d=8, lengthscale=0.5, sf2=1.0, sn2=1e-2, bsz=128, eps=1e-10, seed=1),
    "c2_n131072": dict(N=131072, d=16, lengthscale=1.0, sf2=1.0, sn2=1e-2, bsz=256, eps=1e-10, seed=2),
}


def gp_inputs(N, d, seed, noise_sd=0.1):
    rng = np.random.default_rng(seed)
    X = rng.random((N, d))
    y = np.sin(X.sum(axis=1)) + noise_sd * rng.standard_normal(N)
    return X, y
