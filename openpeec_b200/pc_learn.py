"""Learned correction of the compressed path's preconditioner: training data from the
plain method, training on the GPU, and the weights the sweep takes (pb_sweep_opts.pc_mlp).

The plain preconditioner (precond.c:138-391) LU-factors the leaf-diagonal blocks D_r of
the scaled partial-inductance block and eliminates the circuit unknowns through a dense
Schur complement. The learned part corrects the diagonal of each leaf block,
D_ii <- D_ii (1 + y_i), with y_i = MLP(features of current cell i at wavenumber k). The
target of cell i is (S_r - D_r)_ii / D_ii, where S_r = ((A_LL^-1)_rr)^-1 is the leaf block
that reproduces the diagonal block of the exact inverse of the whole block A_LL
(pb_pc_samples computes it with a dense inverse on the GPU for training-sized structures).
Training is full-batch Adam in the library's own FP32 forward / backward kernels
(pb_mlp_train). The sweep falls back to the plain preconditioner when a prediction is not
finite, when a corrected leaf is singular or when GMRES does not converge with it.
"""
import numpy as np

from . import api, configs, geometry

#: training frequencies: the span of the bar-stack sweep (1 MHz - 2 GHz)
TRAIN_FREQS = (1e6, 1e8, 5e8, 1e9, 2e9)


def plate_family(seed=0, count=6, grid=(6, 16), layers=(2, 4)):
    """Seeded bar stacks of the bar-stack workload's family: 40 x 40 mm plates with
    perturbed side lengths (+-25 %), thickness (0.1 - 0.3 mm) and grids."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        nx, ny = (int(v) for v in rng.integers(grid[0], grid[1] + 1, 2))
        nz = int(rng.integers(layers[0], layers[1] + 1))
        L, W = 0.04 * rng.uniform(0.75, 1.25, 2)
        t = rng.uniform(1e-4, 3e-4)
        text = configs.cfg4(nx, ny, nz, 2, L, W, t)
        out.append(((nx, ny, nz), geometry.build(geometry.parse_peec(text))))
    return out


def collect(problems, freqs=TRAIN_FREQS):
    """Features and targets of every current cell of every structure at every frequency
    (pb_pc_samples). Returns (X [n, 12], T [n, 2]) as float32."""
    X, T = [], []
    for prob in problems:
        with api.Context(prob) as ctx:
            for f in freqs:
                x, t = ctx.pc_samples(f)
                X.append(x)
                T.append(t)
    return np.concatenate(X), np.concatenate(T)


def train(X, T, steps=3000, lr=1e-3, seed=0, want_loss=False):
    """Weights of the correction network trained on (X, T) on the GPU."""
    return api.mlp_train(api.mlp_init(seed), X, T, steps=steps, lr=lr, want_loss=want_loss)
