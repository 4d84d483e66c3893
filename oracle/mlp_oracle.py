"""CPU oracle of the surrogate network's forward and backward passes.

Test infrastructure only: it checks the GPU training kernels' gradients and
is never called by the product path.  It restates, in numpy, the network of
suguru_b200/csrc/sg_surrogate.cu (no counterpart in the reference, whose
membrane force is always the plain model):

  pre_l = h_{l-1} W_l^T + b_l,  h_l = GELU(pre_l) = 0.5 pre (1 + erf(pre/sqrt 2))  (l = 1, 2)
  yhat  = h_2 W_3^T + b_3,      loss = mean((yhat - t)^2)

With emulate_bf16=True it rounds to bf16 at the same points as the kernels
(weights, the stored activations h_{l-1}, and the back-propagated gradients
that enter the products), accumulating every product in float64; with False
it is the exact float64 network, which the finite-difference test pins.
Parameter layout (flat): W1 [dh][din], b1, W2 [dh][dh], b2, W3 [dout][dh], b3.
"""
import numpy as np
from scipy.special import erf


def bf16(x):
    """Round to the nearest bf16 (ties to even), returned as float64."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint32) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def split(params, din, dh, dout):
    sizes = [dh * din, dh, dh * dh, dh, dout * dh, dout]
    shapes = [(dh, din), (dh,), (dh, dh), (dh,), (dout, dh), (dout,)]
    out, o = [], 0
    for n, sh in zip(sizes, shapes):
        out.append(np.asarray(params[o:o + n], dtype=np.float64).reshape(sh))
        o += n
    assert o == params.size
    return out


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def forward_backward(params, X, T, din, dh, dout, emulate_bf16=True):
    """Returns (loss, grads) with grads in the flat parameter layout."""
    q = bf16 if emulate_bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    W1, b1, W2, b2, W3, b3 = split(params, din, dh, dout)
    X = np.asarray(X, dtype=np.float64)
    T = np.asarray(T, dtype=np.float64)
    B = X.shape[0]
    x0 = q(X)
    pre1 = x0 @ q(W1).T + b1
    h1 = q(gelu(pre1))
    pre2 = h1 @ q(W2).T + b2
    h2 = q(gelu(pre2))
    y = h2 @ q(W3).T + b3
    e = y - T
    loss = float(np.mean(e * e))
    dy = 2.0 * e / (B * dout)
    dyq = q(dy)
    gW3 = dyq.T @ h2
    gb3 = dy.sum(0)
    dh2 = dyq @ q(W3)
    dpre2 = dh2 * gelu_grad(pre2)
    dpre2q = q(dpre2)
    gW2 = dpre2q.T @ h1
    gb2 = dpre2.sum(0)
    dh1 = dpre2q @ q(W2)
    dpre1 = dh1 * gelu_grad(pre1)
    gW1 = q(dpre1).T @ x0
    gb1 = dpre1.sum(0)
    grads = np.concatenate([g.ravel() for g in (gW1, gb1, gW2, gb2, gW3, gb3)])
    return loss, grads
