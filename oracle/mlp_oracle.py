"""FP64 restatement of the escape-probability network (TEST INFRASTRUCTURE).

Forward pass, binary cross-entropy loss and its analytic gradient for the
MLP 6 -> 64 -> 64 -> 1 (SiLU hidden, sigmoid output) whose tensor-core
kernels live in nebula_b200/csrc/mlp.cu.  With ``bf16=True`` the operands are
rounded to bfloat16 at the same points as the kernels (inputs, weights,
hidden activations, back-propagated errors) while all arithmetic stays FP64,
so a comparison with the GPU isolates accumulation order and the fast
exponential.  The parameter layout matches include/nbx.h (NBX_MLP_PARAMS).
"""
import numpy as np

F, IN, H, OUT = 6, 16, 64, 8
OFF_W1 = 0
OFF_B1 = OFF_W1 + H * IN
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + OUT * H
N_PARAMS = OFF_B3 + OUT


def bf16(x):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, np.float64)
    W1 = p[OFF_W1:OFF_B1].reshape(H, IN)[:, :F]
    b1 = p[OFF_B1:OFF_W2]
    W2 = p[OFF_W2:OFF_B2].reshape(H, H)
    b2 = p[OFF_B2:OFF_W3]
    W3 = p[OFF_W3:OFF_B3].reshape(OUT, H)[0]
    b3 = p[OFF_B3]
    return W1, b1, W2, b2, W3, b3


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(p, X, emulate_bf16=False):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    r = bf16 if emulate_bf16 else (lambda v: np.asarray(v, np.float64))
    X = r(X)
    z1 = X @ r(W1).T + b1
    h1 = r(silu(z1))
    z2 = h1 @ r(W2).T + b2
    h2 = r(silu(z2))
    logit = h2 @ r(W3) + b3
    return logit, (X, z1, h1, z2, h2)


def predict(p, X, emulate_bf16=False):
    return 1.0 / (1.0 + np.exp(-forward(p, X, emulate_bf16)[0]))


def loss_and_grad(p, X, y, emulate_bf16=False):
    """Mean BCE-with-logits and its gradient (N_PARAMS vector, padding zero)."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    r = bf16 if emulate_bf16 else (lambda v: np.asarray(v, np.float64))
    y = np.asarray(y, np.float64)
    n = len(y)
    logit, (Xr, z1, h1, z2, h2) = forward(p, X, emulate_bf16)
    loss = np.mean(np.logaddexp(0.0, logit) - y * logit)
    pr = 1.0 / (1.0 + np.exp(-logit))
    dz3 = (pr - y) / n
    g = np.zeros(N_PARAMS)
    dz3r = r(dz3)
    g[OFF_W3:OFF_W3 + H] = dz3r @ h2
    g[OFF_B3] = dz3.sum()
    dz2 = (np.outer(dz3r, r(W3))) * silu_grad(z2)
    dz2r = r(dz2)
    g[OFF_W2:OFF_B2] = (dz2r.T @ h1).ravel()
    g[OFF_B2:OFF_W3] = dz2.sum(0)
    dz1 = (dz2r @ r(W2)) * silu_grad(z1)
    dz1r = r(dz1)
    gw1 = np.zeros((H, IN))
    gw1[:, :F] = dz1r.T @ Xr
    g[OFF_W1:OFF_B1] = gw1.ravel()
    g[OFF_B1:OFF_W2] = dz1.sum(0)
    return loss, g


def init_params(seed=0):
    """Seeded Glorot-uniform initialisation with zero biases and zero padding."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, np.float64)
    lim1 = np.sqrt(6.0 / (F + H))
    w1 = np.zeros((H, IN))
    w1[:, :F] = rng.uniform(-lim1, lim1, (H, F))
    p[OFF_W1:OFF_B1] = w1.ravel()
    lim2 = np.sqrt(6.0 / (H + H))
    p[OFF_W2:OFF_B2] = rng.uniform(-lim2, lim2, H * H)
    lim3 = np.sqrt(6.0 / (H + 1))
    p[OFF_W3:OFF_W3 + H] = rng.uniform(-lim3, lim3, H)
    return p.astype(np.float32)
