"""CPU restatement (FP64, numpy) of the per-site dipole-guess network.

Test infrastructure only: the checker of the GPU forward and backward
kernels.  There is no reference code for this network (the reference
starts its dipole solve from p = 1 every step); this file restates the
network the product defines: 24 inputs normalised by the stored mean and
1/std, two tanh layers of 64, 3 outputs, loss (1/(3B)) sum (y - t)^2.
Parameter layout: W1[64][24], b1[64], W2[64][64], b2[64], W3[3][64], b3[3],
then the feature mean[24] and 1/std[24].

With ``bf16=True`` the operands the GPU gives its tensor cores are rounded
to bfloat16 (round to nearest even) at the same places: the normalised
inputs, W1 and W2, h1 as the input of layer 2, and dz2, h1, dz1 and W2 in
the backward products; sums stay in FP64 here (FP32 on the GPU).
"""
import numpy as np

F, H, O = 24, 64, 3
SIZES = [("W1", (H, F)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (O, H)), ("b3", (O,))]
NPARAM = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(params):
    p = np.asarray(params, np.float64)
    out, k = {}, 0
    for name, shp in SIZES:
        n = int(np.prod(shp))
        out[name] = p[k:k + n].reshape(shp)
        k += n
    out["mean"] = p[k:k + F]
    out["istd"] = p[k + F:k + 2 * F]
    return out


def bf(a):
    """float64 -> bfloat16 (round to nearest even) -> float64."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def forward(params, x, bf16=False):
    w = unpack(params)
    if bf16:
        xn = bf((np.asarray(x, np.float32) - w["mean"].astype(np.float32)) * w["istd"].astype(np.float32))
        h1 = np.tanh(xn @ bf(w["W1"]).T + w["b1"])
        h2 = np.tanh(bf(h1) @ bf(w["W2"]).T + w["b2"])
    else:
        xn = (np.asarray(x, np.float64) - w["mean"]) * w["istd"]
        h1 = np.tanh(xn @ w["W1"].T + w["b1"])
        h2 = np.tanh(h1 @ w["W2"].T + w["b2"])
    y = h2 @ w["W3"].T + w["b3"]
    return y, (xn, h1, h2)


def loss_and_grad(params, rows, bf16=False):
    rows = np.asarray(rows, np.float64)
    x, t = rows[:, :F], rows[:, F:F + O]
    w = unpack(params)
    y, (xn, h1, h2) = forward(params, x, bf16)
    B = rows.shape[0]
    e = y - t
    loss = float((e * e).sum() / (3.0 * B))
    dy = 2.0 * e / (3.0 * B)
    g = {"W3": dy.T @ h2, "b3": dy.sum(0)}
    dz2 = (dy @ w["W3"]) * (1.0 - h2 * h2)
    r = bf if bf16 else (lambda a: a)
    g["W2"], g["b2"] = r(dz2).T @ r(h1), dz2.sum(0)
    dz1 = (r(dz2) @ r(w["W2"])) * (1.0 - h1 * h1)
    g["W1"], g["b1"] = r(dz1).T @ xn, dz1.sum(0)
    flat = np.concatenate([g[name].reshape(-1) for name, _ in SIZES])
    return loss, flat
