"""CPU oracle of the learned preconditioner correction's MLP (test infrastructure only:
imported by tests/, never by the library).

The network has no counterpart in the reference; the method it corrects is the leaf-block
+ circuit-Schur preconditioner of precond.c:138-391. This file restates the library's
network in float64 numpy so that the GPU forward pass, the GPU gradient and the GPU Adam
step can be checked against it:

    h1 = tanh(W1 x + b1)        W1 [128, 12]
    h2 = tanh(W2 h1 + b2)       W2 [128, 128]
    y  = W3 h2 + b3             W3 [2, 128]
    L  = mean over samples and outputs of (y - t)^2

Parameters are one flat float32 vector in the order W1, b1, W2, b2, W3, b3 (row-major).
"""
import numpy as np

IN, H, OUT = 12, 128, 2
SHAPES = [(H, IN), (H,), (H, H), (H,), (OUT, H), (OUT,)]
NPARAM = sum(int(np.prod(s)) for s in SHAPES)


def unpack(w):
    w = np.asarray(w, np.float64)
    assert w.size == NPARAM
    out, o = [], 0
    for s in SHAPES:
        k = int(np.prod(s))
        out.append(w[o:o + k].reshape(s))
        o += k
    return out


def forward(w, x):
    W1, b1, W2, b2, W3, b3 = unpack(w)
    x = np.asarray(x, np.float64)
    h1 = np.tanh(x @ W1.T + b1)
    h2 = np.tanh(h1 @ W2.T + b2)
    return h2 @ W3.T + b3, (x, h1, h2)


def loss_grad(w, x, t):
    """Loss and its gradient (flat, float64) by hand-written back-propagation."""
    W1, b1, W2, b2, W3, b3 = unpack(w)
    y, (x, h1, h2) = forward(w, x)
    t = np.asarray(t, np.float64)
    n = len(x)
    d = y - t
    loss = float(np.mean(d * d))
    dy = 2.0 * d / (n * OUT)
    gW3 = dy.T @ h2
    gb3 = dy.sum(0)
    d2 = (dy @ W3) * (1 - h2 * h2)
    gW2 = d2.T @ h1
    gb2 = d2.sum(0)
    d1 = (d2 @ W2) * (1 - h1 * h1)
    gW1 = d1.T @ x
    gb1 = d1.sum(0)
    return loss, np.concatenate([g.ravel() for g in (gW1, gb1, gW2, gb2, gW3, gb3)])


def loss_only(w, x, t):
    y, _ = forward(w, x)
    d = y - np.asarray(t, np.float64)
    return float(np.mean(d * d))


def adam(w, x, t, steps, lr, b1=0.9, b2=0.999, eps=1e-8):
    """Full-batch Adam (Kingma & Ba 2015, bias-corrected), float64."""
    w = np.asarray(w, np.float64).copy()
    m = np.zeros_like(w)
    v = np.zeros_like(w)
    hist = []
    for it in range(1, steps + 1):
        l, g = loss_grad(w, x, t)
        hist.append(l)
        m = b1 * m + (1 - b1) * g
        v = b2 * v + (1 - b2) * g * g
        w -= lr * (m / (1 - b1 ** it)) / (np.sqrt(v / (1 - b2 ** it)) + eps)
    return w, np.array(hist)
