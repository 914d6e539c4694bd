"""CPU oracle of the leaf network (TEST INFRASTRUCTURE ONLY).

Restates the GPU network's forward and backward passes in numpy float64
with BF16 rounding (round to nearest even) at the same points as the GPU:
features, weights, hidden activations and the back-propagated activation
gradients are BF16; products accumulate in high precision; Y, the weight
and bias gradients are FP32.  Used to check the GPU gradients."""
import numpy as np

IN, HID, OUT, INP, OUTP = 2706, 1024, 2652, 2752, 2688


def bf16(x):
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u >> 16) & 1) + 0x7FFF
    return ((u + r) & 0xFFFF0000).astype(np.uint32).view(np.float32).astype(np.float64)


def forward(params, x):
    """params: list of 4 dicts (w [out][in] padded, b [out]); x [M][2706]."""
    M = x.shape[0]
    X0 = np.zeros((M, INP)); X0[:, :IN] = x
    acts = [bf16(X0)]
    h = acts[0]
    for l in range(3):
        z = (h @ bf16(params[l]["w"]).T + params[l]["b"].astype(np.float64)).astype(np.float32)
        h = bf16(np.maximum(z, 0.0))
        acts.append(h)
    y = (h @ bf16(params[3]["w"]).T + params[3]["b"].astype(np.float64)).astype(np.float32)
    return acts, y


def gradients(params, x, t, w=None):
    """Masked MSE sum(w (y - t)^2) / (M * 2652) and its gradients per layer."""
    M = x.shape[0]
    acts, y = forward(params, x)
    T = np.zeros((M, OUTP)); T[:, :OUT] = t
    W = np.zeros((M, OUTP)); W[:, :OUT] = 1.0 if w is None else w
    n = M * OUT
    d = y.astype(np.float64) - T
    loss = float((W * d * d).sum() / n)
    g = bf16((2.0 * W * d / n).astype(np.float32))
    grads = [None] * 4
    for l in range(3, -1, -1):
        gw = (g.T @ acts[l]).astype(np.float32)
        gb = g.sum(axis=0).astype(np.float32)
        grads[l] = {"gw": gw, "gb": gb}
        if l == 0:
            break
        dh = (g @ bf16(params[l]["w"])).astype(np.float32)
        g = bf16(np.where(acts[l] > 0, dh, 0.0))
    return loss, y, grads
