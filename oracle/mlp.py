"""CPU restatement of the learned preconditioner's perceptron (numpy, FP64).

TEST INFRASTRUCTURE: only tests/ use this module, as the checker of the
device kernels in gecco-public_b200/csrc/learned.cu (inputs, corrected step,
loss and its gradient with respect to the weights).  It restates the same
definitions; the reference has no counterpart (its step is diavc,
baserout/diavc.f:31-35).

Weights (1217 doubles): W1[32][3], b1[32], W2[32][32], b2[32], W3[32], b3.
Inputs of an element with d = diag + shift (|d| <= 1e-10 -> 1e-10), plain
step s = fac*in/d, previous step p:
  x0 = d/4, x1 = 1/max(|d|, 0.05), x2 = clip((s/rms(s)) * (p/rms(p)), -10, 10)
Output o = W3 . tanh(W2 tanh(W1 x + b1) + b2) + b3; corrected step
s*(1 + tanh(o)); loss over rows (x, s, target): mean (s*(1+tanh o) - target)^2.
"""
import numpy as np

NI, NH = 3, 32
NW = NH * NI + NH + NH * NH + NH + NH + 1


def unpack(w):
    w = np.asarray(w, dtype=np.float64)
    assert w.size == NW
    o = 0
    W1 = w[o:o + NH * NI].reshape(NH, NI); o += NH * NI
    b1 = w[o:o + NH]; o += NH
    W2 = w[o:o + NH * NH].reshape(NH, NH); o += NH * NH
    b2 = w[o:o + NH]; o += NH
    W3 = w[o:o + NH]; o += NH
    b3 = w[o]
    return W1, b1, W2, b2, W3, b3


def init_weights(seed, out_scale=0.01):
    rng = np.random.default_rng(seed)
    W1 = rng.normal(0.0, 1.0 / np.sqrt(NI), (NH, NI))
    W2 = rng.normal(0.0, 1.0 / np.sqrt(NH), (NH, NH))
    W3 = rng.normal(0.0, out_scale, NH)
    return np.concatenate([W1.ravel(), np.zeros(NH), W2.ravel(), np.zeros(NH), W3, [0.0]])


def denom(diag, shift=0.0):
    d = np.asarray(diag, dtype=np.float64) + shift
    return np.where(np.abs(d) <= 1e-10, 1e-10, d)


def inputs(inp, diag, prev, fac=1.0, shift=0.0):
    """(x[n,3], s[n]) of whole lists"""
    d = denom(diag, shift)
    s = fac * np.asarray(inp) / d
    ms = np.mean(s * s)
    u = s / np.sqrt(ms) if ms > 0 else np.zeros_like(s)
    if prev is None:
        v = np.zeros_like(s)
    else:
        mp = np.mean(np.asarray(prev) ** 2)
        v = np.asarray(prev) / np.sqrt(mp) if mp > 0 else np.zeros_like(s)
    x = np.stack([d / 4.0, 1.0 / np.maximum(np.abs(d), 0.05), np.clip(u * v, -10.0, 10.0)], 1)
    return x, s


def forward(w, x):
    W1, b1, W2, b2, W3, b3 = unpack(w)
    h1 = np.tanh(x @ W1.T + b1)
    h2 = np.tanh(h1 @ W2.T + b2)
    return h2 @ W3 + b3, (h1, h2)


def step(w, inp, diag, prev, fac=1.0, shift=0.0):
    x, s = inputs(inp, diag, prev, fac, shift)
    o, _ = forward(w, x)
    return s * (1.0 + np.tanh(o))


def loss_and_gradient(w, x, s, target):
    """L = mean (s (1 + tanh o) - target)^2 and dL/dw (packed like w)"""
    W1, b1, W2, b2, W3, b3 = unpack(w)
    n = len(s)
    o, (h1, h2) = forward(w, x)
    c = np.tanh(o)
    r = s * (1.0 + c) - target
    L = np.sum(r * r) / n
    do = 2.0 * r * s * (1.0 - c * c) / n
    gW3 = h2.T @ do
    gb3 = np.sum(do)
    d2 = do[:, None] * W3[None, :] * (1.0 - h2 * h2)
    gW2 = d2.T @ h1
    gb2 = d2.sum(0)
    d1 = (d2 @ W2) * (1.0 - h1 * h1)
    gW1 = d1.T @ x
    gb1 = d1.sum(0)
    return L, np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3, [gb3]])
