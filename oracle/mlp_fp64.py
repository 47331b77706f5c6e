"""FP64 restatement of the learned proposals' network.  TEST INFRASTRUCTURE ONLY.

The network of vapoursynth-vnlb_b200/csrc/learned.cu in float64 numpy:
layers of x W_l^T + b_l with ReLU on the hidden layers, softmax
cross-entropy against up to tk target classes per row (-1 = none), each
weighted 1 / (their count), averaged over the rows.  The forward products use
the weights rounded to BF16 (round to nearest even), as the CUDA kernels do;
the gradients are those of that function.  `numeric_gradients` checks the
analytical ones by central differences.  Weights are flat, layer by layer
[W_l (fan_out x fan_in)][b_l].
"""
from __future__ import annotations

import numpy as np


def bf16(w: np.ndarray) -> np.ndarray:
    """float32 -> the nearest BF16 value (ties to even), as float64."""
    u = np.ascontiguousarray(w, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(flat: np.ndarray, inputs: int, hidden: int, layers: int, outputs: int):
    ws, bs, off = [], [], 0
    for l in range(layers + 1):
        fi = inputs if l == 0 else hidden
        fo = outputs if l == layers else hidden
        ws.append(np.asarray(flat[off:off + fo * fi], np.float64).reshape(fo, fi))
        off += fo * fi
        bs.append(np.asarray(flat[off:off + fo], np.float64))
        off += fo
    return ws, bs


def forward_logits(flat, shape, x, bf16_last_input=False):
    """Logits in float64 with the BF16-rounded weights; bf16_last_input
    also rounds the output layer's input activations to BF16, as the
    tensor-core inference does (learned.cu, tc_logits_kernel)."""
    inputs, hidden, layers, outputs = shape
    ws, bs = unpack(flat, *shape)
    a = np.asarray(x, np.float64)
    for l in range(layers):
        a = np.maximum(a @ bf16(ws[l].astype(np.float32)).T + bs[l], 0.0)
    if bf16_last_input:
        a = bf16(a.astype(np.float32))
    return a @ bf16(ws[layers].astype(np.float32)).T + bs[layers]


def loss_and_gradients(flat, shape, x, targets, round_weights=True):
    """(mean loss, flat gradients) in float64."""
    inputs, hidden, layers, outputs = shape
    ws, bs = unpack(flat, *shape)
    wf = [bf16(w.astype(np.float32)) if round_weights else w for w in ws]
    x = np.asarray(x, np.float64)
    acts = [x]
    for l in range(layers):
        acts.append(np.maximum(acts[-1] @ wf[l].T + bs[l], 0.0))
    z = acts[-1] @ wf[layers].T + bs[layers]
    rows = x.shape[0]
    zmax = z.max(axis=1, keepdims=True)
    lse = zmax + np.log(np.exp(z - zmax).sum(axis=1, keepdims=True))
    target = np.zeros_like(z)
    for r in range(rows):
        valid = [t for t in targets[r] if 0 <= t < outputs]
        for t in valid:
            target[r, t] += 1.0 / len(valid)
    loss = float(((lse - z) * target).sum() / rows)
    grad = (np.exp(z - lse) - target) / rows
    gws, gbs = [None] * (layers + 1), [None] * (layers + 1)
    for l in range(layers, -1, -1):
        gws[l] = grad.T @ acts[l]
        gbs[l] = grad.sum(axis=0)
        if l == 0:
            break
        grad = (grad @ wf[l]) * (acts[l] > 0.0)
    flat_g = np.concatenate([np.concatenate([gw.reshape(-1), gb]) for gw, gb in zip(gws, gbs)])
    return loss, flat_g


def numeric_gradients(flat, shape, x, targets, indices, h=1e-6):
    """Central differences of the mean loss (weights not rounded) at `indices`."""
    flat = np.asarray(flat, np.float64)
    out = []
    for i in indices:
        p, m = flat.copy(), flat.copy()
        p[i] += h
        m[i] -= h
        out.append((loss_and_gradients(p, shape, x, targets, False)[0] -
                    loss_and_gradients(m, shape, x, targets, False)[0]) / (2 * h))
    return np.array(out)
