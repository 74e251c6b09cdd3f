"""numpy restatement of the exchange control-variate MLP (test infrastructure only).

Forward and backward of ``16 -> H -> H -> 1`` with SiLU activations and an MSE
loss, in float64, with the weight matrices rounded to bf16 exactly as the
CUDA forward kernels read them (biases stay fp32).  Used by the tests to check
the GPU kernels' gradients; nothing in ``ipie_b200`` imports it.
"""
import numpy as np


def bf16_round(x):
    """Round float32 values to bfloat16 (round to nearest even), returned as float64."""
    f = np.ascontiguousarray(np.asarray(x, dtype=np.float32)).view(np.uint32)
    bias = ((f >> 16) & 1) + np.uint32(0x7FFF)
    return ((f + bias) & np.uint32(0xFFFF0000)).view(np.float32).astype(np.float64)


def unpack(theta, F, H):
    o = 0
    W1 = theta[o:o + F * H].reshape(F, H); o += F * H
    b1 = theta[o:o + H]; o += H
    W2 = theta[o:o + H * H].reshape(H, H); o += H * H
    b2 = theta[o:o + H]; o += H
    W3 = theta[o:o + H].reshape(H, 1); o += H
    b3 = theta[o:o + 1]
    return W1, b1, W2, b2, W3, b3


def silu(a):
    return a / (1.0 + np.exp(-a))


def silu_grad(a):
    s = 1.0 / (1.0 + np.exp(-a))
    return s * (1.0 + a * (1.0 - s))


def forward(x, theta, F, H):
    W1, b1, W2, b2, W3, b3 = unpack(np.asarray(theta, dtype=np.float64), F, H)
    W1, W2, W3 = bf16_round(W1), bf16_round(W2), bf16_round(W3)
    a1 = x @ W1 + b1
    h1 = silu(a1)
    a2 = h1 @ W2 + b2
    h2 = silu(a2)
    out = (h2 @ W3 + b3)[:, 0]
    return out, (a1, h1, a2, h2)


def mse_grad(x, y, theta, F, H):
    """Loss and gradient of mean((out - y)^2) with respect to the packed parameters."""
    W1, b1, W2, b2, W3, b3 = unpack(np.asarray(theta, dtype=np.float64), F, H)
    W1b, W2b, W3b = bf16_round(W1), bf16_round(W2), bf16_round(W3)
    out, (a1, h1, a2, h2) = forward(x, theta, F, H)
    B = x.shape[0]
    d = out - y
    loss = np.mean(d * d)
    dout = (2.0 * d / B)[:, None]
    gW3 = h2.T @ dout
    gb3 = dout.sum(0)
    dh2 = (dout @ W3b.T) * silu_grad(a2)
    gW2 = h1.T @ dh2
    gb2 = dh2.sum(0)
    dh1 = (dh2 @ W2b.T) * silu_grad(a1)
    gW1 = x.T @ dh1
    gb1 = dh1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g
