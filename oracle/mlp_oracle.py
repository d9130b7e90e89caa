"""CPU oracle of the learned limiter's MLP (numpy): TEST INFRASTRUCTURE ONLY.

Restates luna_cpp_b200/csrc/hydro/mlp.cuh's forward and backward with the same roundings to BF16 (weights, activations
and the backward's MMA inputs; FP32 accumulation), so the tests can check the tensor-core kernels' logits and gradients.
The network has no counterpart in the reference.
"""
import numpy as np

IN, HID, OUT, USED = 32, 64, 16, 5
W1, B1 = 0, HID * IN
W2 = B1 + HID
B2 = W2 + HID * HID
W3 = B2 + HID
B3 = W3 + OUT * HID
PARAMS = B3 + OUT


def bf16(a):
    """float32 -> bfloat16 (round to nearest even), returned as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32).reshape(a.shape)


def unpack(p):
    p = np.asarray(p, dtype=np.float32)
    return (p[W1:B1].reshape(HID, IN), p[B1:W2], p[W2:B2].reshape(HID, HID), p[B2:W3], p[W3:B3].reshape(OUT, HID),
            p[B3:PARAMS])


def forward(p, x):
    w1, b1, w2, b2, w3, b3 = unpack(p)
    x = bf16(x)
    h1 = np.maximum(x @ bf16(w1).T + b1, 0).astype(np.float32)
    h2 = np.maximum(bf16(h1) @ bf16(w2).T + b2, 0).astype(np.float32)
    out = (bf16(h2) @ bf16(w3).T + b3).astype(np.float32)
    return out, (x, h1, h2)


def loss_and_grad(p, x, target, weight, scale):
    w1, b1, w2, b2, w3, b3 = unpack(p)
    out, (xb, h1, h2) = forward(p, x)
    sg = 1.0 / (1.0 + np.exp(-out[:, :USED]))
    e = sg - target
    loss = float(np.sum(weight * e * e)) * scale
    dout = np.zeros_like(out)
    dout[:, :USED] = 2 * weight * e * sg * (1 - sg)
    doutb = bf16(dout)
    dz2 = doutb @ bf16(w3)
    dz2[h2 <= 0] = 0
    dz2b = bf16(dz2)
    dz1 = dz2b @ bf16(w2)
    dz1[h1 <= 0] = 0
    dz1b = bf16(dz1)
    g = np.zeros(PARAMS, dtype=np.float64)
    g[W1:B1] = (dz1b.T.astype(np.float64) @ xb).ravel()
    g[B1:W2] = dz1b.sum(0)
    g[W2:B2] = (dz2b.T.astype(np.float64) @ bf16(h1)).ravel()
    g[B2:W3] = dz2b.sum(0)
    g[W3:B3] = (doutb.T.astype(np.float64) @ bf16(h2)).ravel()
    g[B3:PARAMS] = doutb.sum(0)
    return loss, (g * scale).astype(np.float32)
