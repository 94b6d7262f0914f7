"""Reference (numpy, FP64) forward and backward pass of the learned order selector's network
-- TEST INFRASTRUCTURE ONLY, the checker of the hand-written CUDA kernels in
taichi_collisional_b200/csrc/tc_mlp.cuh (k_mlp_grad, k_mlp_predict).

Layout of the parameter vector: W1[32][8] b1[32] W2[32][32] b2[32] W3[32][32] b3[32]
W4[nout][32] b4[nout]; tanh hidden layers; loss = mean over samples and outputs of
(y - (label - out_mean))^2 with standardised inputs (x - mean) * inv_std.
"""
import numpy as np

H, IN = 32, 8


def unpack(w, nout):
    w = np.asarray(w, dtype=np.float64)
    o = 0
    out = []
    for shape in ((H, IN), (H,), (H, H), (H,), (H, H), (H,), (nout, H), (nout,)):
        size = int(np.prod(shape))
        out.append(w[o:o + size].reshape(shape))
        o += size
    assert o == len(w)
    return out


def forward(w, nout, feat, norm):
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(w, nout)
    x = (np.asarray(feat, np.float64) - norm[:IN]) * norm[IN:2 * IN]
    a1 = np.tanh(x @ W1.T + b1)
    a2 = np.tanh(a1 @ W2.T + b2)
    a3 = np.tanh(a2 @ W3.T + b3)
    y = a3 @ W4.T + b4
    return x, a1, a2, a3, y


def predict(w, nout, feat, norm):
    return forward(w, nout, feat, norm)[-1] + norm[2 * IN]


def loss_grad(w, nout, feat, labels, norm):
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(w, nout)
    x, a1, a2, a3, y = forward(w, nout, feat, norm)
    ns = len(x)
    e = y - (np.asarray(labels, np.float64) - norm[2 * IN])
    loss = (e * e).mean()
    d4 = 2.0 * e / (ns * nout)
    gW4 = d4.T @ a3
    gb4 = d4.sum(0)
    d3 = (d4 @ W4) * (1 - a3 * a3)
    gW3 = d3.T @ a2
    gb3 = d3.sum(0)
    d2 = (d3 @ W3) * (1 - a2 * a2)
    gW2 = d2.T @ a1
    gb2 = d2.sum(0)
    d1 = (d2 @ W2) * (1 - a1 * a1)
    gW1 = d1.T @ x
    gb1 = d1.sum(0)
    g = np.concatenate([a.ravel() for a in (gW1, gb1, gW2, gb2, gW3, gb3, gW4, gb4)])
    return loss, g
