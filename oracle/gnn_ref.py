"""FP64 numpy restatement of the learned stepper's message-passing network:
forward pass, loss and analytic backward pass.  TEST INFRASTRUCTURE ONLY:
tests use it as the checker of the GPU network (bf16 tensor-core GEMMs,
fp32 accumulation); nothing in the product imports it.  It has no
counterpart in the reference, whose step is the SPH solver alone; its own
correctness is pinned by central finite differences in the CPU tests.

Network (L = latent width, s = aggregation scale, relu(t) = max(t, 0)):
    h = W2n relu(W1n fn + b1n) + b2n                       node encoder
    e = W2e relu(W1e fe + b1e) + b2e                       edge encoder
    per layer:
        P   = h Wsd^T                                      [Ws; Wd] stacked
        z   = e We^T + P[src, :L] + P[dst, L:] + be
        e   = e + relu(z) W2^T + b2                        edge update
        agg = s * sum of e over the edges each node receives
        y   = [h, agg] V1^T + c1
        h   = h + relu(y) V2^T + c2                        node update
    out = D2 relu(D1 h + d1) + d2;  prediction = out[:, :2]
    loss = sum over masked rows and 2 columns of (pred - target)^2 / (2 * rows)
Weights are stored as [out x in] matrices; names follow weight_names().
"""
from __future__ import annotations

import numpy as np


def weight_names(layers: int):
    w = ["enc_n.w1", "enc_n.w2", "enc_e.w1", "enc_e.w2"]
    b = ["enc_n.b1", "enc_n.b2", "enc_e.b1", "enc_e.b2"]
    for l in range(layers):
        w += [f"p{l}.we", f"p{l}.wsd", f"p{l}.w2", f"p{l}.v1", f"p{l}.v2"]
        b += [f"p{l}.be", f"p{l}.b2", f"p{l}.c1", f"p{l}.c2"]
    return w + ["dec.w1", "dec.w2"], b + ["dec.b1", "dec.b2"]


def _relu(t):
    return np.maximum(t, 0.0)


def bf16(a):
    """Round to bfloat16 (through float32, round to nearest even), as FP64."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32).astype(np.float64)


def _ident(a):
    return a


def forward(W, fn, fe, src, dst, n_nodes, layers, scale, keep=True, round_bf16=False):
    """Returns (out, cache); fn [n, F], fe [e, F].  With round_bf16 every
    matrix-product operand is rounded to bfloat16 where the GPU network
    rounds it (weights are taken as given)."""
    q = bf16 if round_bf16 else _ident
    c = {}
    L = W["enc_n.w2"].shape[0]
    nz = q(fn) @ W["enc_n.w1"].T + W["enc_n.b1"]
    h = q(_relu(nz)) @ W["enc_n.w2"].T + W["enc_n.b2"]
    ez = q(fe) @ W["enc_e.w1"].T + W["enc_e.b1"]
    e = q(_relu(ez)) @ W["enc_e.w2"].T + W["enc_e.b2"]
    c["nz"], c["ez"] = nz, ez
    for l in range(layers):
        p = f"p{l}."
        c[p + "h"], c[p + "e"] = q(h), q(e)
        P = q(h) @ W[p + "wsd"].T
        z = q(e) @ W[p + "we"].T + P[src, :L] + P[dst, L:] + W[p + "be"]
        e = e + q(_relu(z)) @ W[p + "w2"].T + W[p + "b2"]
        agg = np.zeros((n_nodes, L))
        np.add.at(agg, dst, e)
        agg *= scale
        cat = np.concatenate([q(h), q(agg)], axis=1)
        y = cat @ W[p + "v1"].T + W[p + "c1"]
        h = h + q(_relu(y)) @ W[p + "v2"].T + W[p + "c2"]
        c[p + "z"], c[p + "cat"], c[p + "y"] = z, cat, y
    u = q(h) @ W["dec.w1"].T + W["dec.b1"]
    out = q(_relu(u)) @ W["dec.w2"].T + W["dec.b2"]
    c["hL"], c["u"] = q(h), u
    c["q"] = q
    return out, c


def loss_and_grad_out(out, target, mask, nout=2, delta=0.0):
    """Masked mean squared error over the first nout columns; with delta > 0
    the Huber form (linear beyond |d| = delta)."""
    rows = mask != 0
    count = float(rows.sum() * nout)
    d = out[:, :nout] - target
    d[~rows] = 0.0
    g = np.zeros_like(out)
    if delta > 0:
        a = np.abs(d)
        lin = a > delta
        val = np.where(lin, delta * (2 * a - delta), d * d)
        g[:, :nout] = np.where(lin, 2.0 * delta * np.sign(d), 2.0 * d) / count
        return float(val.sum() / count), g
    g[:, :nout] = 2.0 * d / count
    return float((d * d).sum() / count), g


def decoder_backward(W, dout, u, hL, q):
    """Decoder stage: gradients of dec.* and of the last node state."""
    G = {}
    qo = q(dout)
    G["dec.w2"] = qo.T @ q(_relu(u))
    G["dec.b2"] = dout.sum(0)
    du = (qo @ W["dec.w2"]) * (u > 0)
    G["dec.w1"] = q(du).T @ hL
    G["dec.b1"] = du.sum(0)
    return G, q(du) @ W["dec.w1"]


def layer_backward(W, p, dh, de, h, e, z, cat, y, src, dst, n_nodes, scale, q):
    """One message-passing layer: gradients of its weights and of its input
    node and edge states, given those of its outputs (h, e: the layer's
    rounded inputs; z, cat, y: its saved pre-activations and concatenation)."""
    G = {}
    L = h.shape[1]
    # node update
    G[p + "c2"] = dh.sum(0)
    G[p + "v2"] = q(dh).T @ q(_relu(y))
    dy = (q(dh) @ W[p + "v2"]) * (y > 0)
    G[p + "c1"] = dy.sum(0)
    G[p + "v1"] = q(dy).T @ cat
    dcat = q(dy) @ W[p + "v1"]
    dh = dh + dcat[:, :L]
    de = de + scale * dcat[dst, L:]
    # edge update
    G[p + "b2"] = de.sum(0)
    G[p + "w2"] = q(de).T @ q(_relu(z))
    dz = (q(de) @ W[p + "w2"]) * (z > 0)
    G[p + "be"] = dz.sum(0)
    G[p + "we"] = q(dz).T @ e
    de = de + q(dz) @ W[p + "we"]
    dP = np.zeros((n_nodes, 2 * L))
    np.add.at(dP[:, :L], src, dz)
    np.add.at(dP[:, L:], dst, dz)
    G[p + "wsd"] = q(dP).T @ h
    dh = dh + q(dP) @ W[p + "wsd"]
    return G, dh, de


def encoder_backward(W, dh, de, nz, ez, fn, fe, q):
    G = {}
    for side, d, z, f in (("n", dh, nz, fn), ("e", de, ez, fe)):
        enc = "enc_" + side
        G[enc + ".b2"] = d.sum(0)
        G[enc + ".w2"] = q(d).T @ q(_relu(z))
        dz = (q(d) @ W[enc + ".w2"]) * (z > 0)
        G[enc + ".b1"] = dz.sum(0)
        G[enc + ".w1"] = q(dz).T @ q(f)
    return G


def backward(W, fn, fe, src, dst, n_nodes, layers, scale, cache, dout):
    """Gradients of every weight and bias given d loss / d out (rounding the
    matrix-product operands as the forward pass of the cache did), plus
    "_dh0" and "_de0", the gradients of the encoded node and edge states."""
    q = cache["q"]
    L = W["enc_n.w2"].shape[0]
    G, dh = decoder_backward(W, dout, cache["u"], cache["hL"], q)
    de = np.zeros((len(src), L))
    for l in reversed(range(layers)):
        p = f"p{l}."
        g, dh, de = layer_backward(W, p, dh, de, *(cache[p + k] for k in ("h", "e", "z", "cat", "y")), src, dst,
                                   n_nodes, scale, q)
        G.update(g)
    G["_dh0"], G["_de0"] = dh, de
    G.update(encoder_backward(W, dh, de, cache["nz"], cache["ez"], fn, fe, q))
    return G


def radius_graph(x, radius):
    """Every ordered pair (src, dst), dst != src, closer than radius, grouped
    by receiver (dst ascending) then sender ascending: a brute-force O(n^2)
    reference for small node counts."""
    d2 = ((x[:, None, :] - x[None, :, :]) ** 2).sum(-1)
    dst, src = np.nonzero(d2 < radius * radius)
    keep = dst != src
    return src[keep].astype(np.int64), dst[keep].astype(np.int64)
