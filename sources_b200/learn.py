"""Learned particle stepper: a message-passing network over the particles
that predicts each particle's mean acceleration over a stride of k solver
steps, trained on rollouts of the batched SPH solver, with the plain SPH
step as its fallback and as the yardstick of its error.  The reference has no
counterpart: its step is the SPH solver alone.

Everything numeric runs in libsphg's own CUDA kernels (include/sphg_learn.h):
the dense layers on the tcgen05 BF16 GEMM (fp32 accumulation in TMEM), the
graph search, features, gathers, scatters, segment sums, loss, Adam and the
stride update in sphg_gnn.cu.  PyTorch only allocates device memory, copies
buffers and assembles training batches (indexing and noise).

Network (latent width L = 128, 4 message-passing layers, 2-layer MLPs):
    node inputs  5 velocities (newest first), type one-hot (water, soil,
                 boundary), wall distances / 2h clipped to [0, 1], porosity,
                 friction angle, stride length   (19 of 64 padded columns)
    edge inputs  (x_receiver - x_sender) / 2h, distance / 2h, same-type flag
    edges        every pair closer than 2h, both directions
    encoder      2-layer MLPs to L for nodes and edges
    layer        z = e We^T + h[src] Ws^T + h[dst] Wd^T + be   (the [e, h_src,
                 h_dst] input of the edge MLP, with the node projections
                 computed once per node and gathered per edge);
                 e += relu(z) W2^T + b2;  agg = sum of e over received edges / 16;
                 h += relu([h, agg] V1^T + c1) V2^T + c2
    decoder      2-layer MLP to the 2 acceleration components (normalised)
Velocities are finite differences over a stride, v_t = (x_t - x_{t-k}) / D
with D = k dt (k = 10 solver steps of the scene's dt), and the target is the
stride acceleration a_t = (x_{t+k} - 2 x_t + x_{t-k}) / D^2: position
differences average out the acoustic oscillations that the solver's own
velocities carry at a period of a few steps.  Stride update (semi-implicit
Euler, exact for the exact a): v' = v + a D, x' = x + v' D, clamped inside
the walls.  Fallback gates: the
RMS relative change of the SPH number density over real particles above
1 %, or a rise of kinetic + potential energy above 5 % of (kinetic energy +
one dx of potential energy per particle); a failed stride is redone by k
plain SPH steps.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import time
from dataclasses import dataclass, field

import numpy as np

from . import SPHError, load
from .abi import SPHG_SOIL, SPHG_WATER

L_WIDTH = 128
F_IN = 64
LAYERS = 4
AGG_SCALE = 1.0 / 16.0
NOUT = 2
K_STRIDE = 10
HIST = 5
GRAVITY = -9.800000190734863     # the solver's default gravity (single-precision -9.8)
GATE_DENSITY = 0.01
GATE_ENERGY = 0.05
TARGET_CLAMP = 20.0      # normalised acceleration targets, in std
HUBER_DELTA = 3.0        # training loss: squared error up to 3 std, linear beyond

GNN_WATER, GNN_SOIL, GNN_BOUNDARY = 0, 1, 2
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "learned_weights.npz")
NODE_DTYPE = np.dtype([("xl", "<f4"), ("xr", "<f4"), ("yf", "<f4"), ("dts", "<f4"), ("porosity", "<f4"),
                       ("phi", "<f4"), ("mass", "<f4"), ("type", "<i4")])


class GemmEpi(C.Structure):
    """SphgGemmEpi (include/sphg_learn.h): the fused epilogue of the
    weight-stationary GEMM."""
    _fields_ = [("mode", C.c_int32), ("relu", C.c_int32), ("bias", C.c_void_p), ("z", C.c_void_p),
                ("h", C.c_void_p), ("P", C.c_void_p), ("src", C.c_void_p), ("dst", C.c_void_p),
                ("nedge", C.c_longlong)]


EPI_STORE, EPI_ACC, EPI_BIAS_ACT, EPI_EDGE, EPI_RESID = range(5)


class Grid(C.Structure):
    _fields_ = [("xmin", C.c_double), ("ymin", C.c_double), ("radius", C.c_double), ("nx", C.c_int32),
                ("ny", C.c_int32)]


def pad128(n: int) -> int:
    return max(128, (n + 127) // 128 * 128)


def weight_specs():
    """[(name, rows, cols, row_limit)] of the weights, [(name, size, limit)] of the biases."""
    L, F = L_WIDTH, F_IN
    W = [("enc_n.w1", L, F), ("enc_n.w2", L, L), ("enc_e.w1", L, F), ("enc_e.w2", L, L)]
    B = ["enc_n.b1", "enc_n.b2", "enc_e.b1", "enc_e.b2"]
    for l in range(LAYERS):
        W += [(f"p{l}.we", L, L), (f"p{l}.wsd", 2 * L, L), (f"p{l}.w2", L, L), (f"p{l}.v1", L, 2 * L),
              (f"p{l}.v2", L, L)]
        B += [f"p{l}.be", f"p{l}.b2", f"p{l}.c1", f"p{l}.c2"]
    W += [("dec.w1", L, L), ("dec.w2", L, L)]
    B += ["dec.b1", "dec.b2"]
    lim = {"dec.w2": NOUT, "dec.b2": NOUT}
    return ([(n, r, c, lim.get(n, r)) for n, r, c in W], [(n, L, lim.get(n, L)) for n in B])


def init_weights(seed: int = 0) -> dict:
    """Uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights, zero biases (PCG64 seed)."""
    g = np.random.Generator(np.random.PCG64(seed))
    out = {}
    Ws, Bs = weight_specs()
    for name, r, c, lim in Ws:
        a = 1.0 / math.sqrt(c)
        w = g.uniform(-a, a, size=(r, c)).astype(np.float32)
        w[lim:] = 0.0
        out[name] = w
    for name, r, lim in Bs:
        out[name] = np.zeros(r, np.float32)
    return out


def _torch():
    import torch
    return torch


def _ptr(t) -> int:
    return 0 if t is None else t.data_ptr()


def _call(rc: int, what: str):
    if rc != 0:
        raise SPHError(rc, what)


class _Buffers:
    """Grow-only named device buffers; new memory is zeroed, so every view
    holds finite values."""

    def __init__(self, device):
        self.torch = _torch()
        self.device = device
        self.buf = {}

    def get(self, name, shape, dtype, zero=False):
        numel = int(np.prod(shape))
        t = self.buf.get(name)
        if t is None or t.numel() < numel:
            # a quarter of headroom when a buffer grows, so that graphs growing by a few
            # edges from stride to stride do not reallocate (and zero) every time
            grown = numel if t is None else numel + numel // 4
            t = self.torch.zeros(max(grown, 1), dtype=dtype, device=self.device)
            self.buf[name] = t
        v = t[:numel].view(*shape)
        if zero:
            v.zero_()
        return v


@dataclass
class Batch:
    """One graph on the device: n nodes (rows padded to n_pad), E edges."""
    n: int
    n_pad: int
    E: int
    E_pad: int
    x: object            # [n, 2] f64
    nodes: object        # [n, 32] uint8 (NODE_DTYPE rows)
    off: object          # [n + 1] int64
    src: object          # [E] int32
    dst: object
    fn: object           # [n_pad, 64] bf16
    fe: object           # [E_pad, 64] bf16
    target: object = None
    mask: object = None
    n_real: int = 0


class GraphBuilder:
    """Radius graph of the particles on the device (sphg_gnn_graph_count /
    _fill): the edge count is read back once to size the edge arrays."""

    def __init__(self, lib, bufs: _Buffers, prefix="g"):
        self.L, self.b, self.p = lib, bufs, prefix
        self.torch = bufs.torch

    def build(self, x, n: int, grid: Grid, stream: int):
        t = self.torch
        ncell = grid.nx * grid.ny
        nbytes = C.c_size_t()
        _call(self.L.sphg_gnn_scan_bytes(max(ncell, n), C.byref(nbytes)), "sphg_gnn_scan_bytes")
        tmp = self.b.get(self.p + ".tmp", (nbytes.value + 16,), t.uint8)
        order = self.b.get(self.p + ".order", (n,), t.int32)
        cc = self.b.get(self.p + ".cc", (ncell + 1,), t.int32)
        cs = self.b.get(self.p + ".cs", (ncell + 1,), t.int32)
        deg = self.b.get(self.p + ".deg", (n + 1,), t.int32)
        off = self.b.get(self.p + ".off", (n + 1,), t.int64)
        _call(self.L.sphg_gnn_graph_count(C.byref(grid), _ptr(x), n, _ptr(order), _ptr(cc), _ptr(cs), _ptr(deg),
                                          _ptr(off), _ptr(tmp), nbytes.value, stream), "sphg_gnn_graph_count")
        E = int(off[n].item())
        if E < 0 or E >= 2 ** 31 - 1:
            raise SPHError(4, "graph edge count out of range")
        src = self.b.get(self.p + ".src", (max(E, 1),), t.int32)
        dst = self.b.get(self.p + ".dst", (max(E, 1),), t.int32)
        _call(self.L.sphg_gnn_graph_fill(C.byref(grid), _ptr(x), n, _ptr(order), _ptr(cs), _ptr(off), _ptr(src),
                                         _ptr(dst), stream), "sphg_gnn_graph_fill")
        return off, src, dst, E


class MPNet:
    """The message-passing network with its device weights, Adam state and
    activation buffers; forward/backward call libsphg kernels only."""

    def __init__(self, weights: dict | None = None, seed: int = 0, device="cuda"):
        self.torch = t = _torch()
        self.L = load()
        self.device = t.device(device)
        self.bufs = _Buffers(self.device)
        self.graph = GraphBuilder(self.L, self.bufs)
        w = weights if weights is not None else init_weights(seed)
        self.W, self.B = {}, {}
        Ws, Bs = weight_specs()
        for name, r, c, lim in Ws:
            m = t.from_numpy(np.ascontiguousarray(w[name], dtype=np.float32)).to(self.device)
            self.W[name] = dict(w=m, wb=m.to(t.bfloat16), wt=m.t().contiguous().to(t.bfloat16), g=t.zeros_like(m),
                                m=t.zeros_like(m), v=t.zeros_like(m), rows=r, cols=c, lim=lim)
        for name, r, lim in Bs:
            m = t.from_numpy(np.ascontiguousarray(w[name], dtype=np.float32)).to(self.device)
            self.B[name] = dict(w=m, g=t.zeros_like(m), m=t.zeros_like(m), v=t.zeros_like(m), rows=r, lim=lim)
        self.err = t.zeros(1, dtype=t.int32, device=self.device)
        self.loss_buf = t.zeros(1, dtype=t.float32, device=self.device)
        self.adam_step = 0
        # inputs include the displacement since the reference positions
        self.use_x0 = True
        # normalisation: velocity scale, acceleration mean (2) and std (2)
        self.vscale = 1.0
        self.norm = t.tensor([0.0, 0.0, 1.0, 1.0], dtype=t.float32, device=self.device)
        self.launches = 0
        # inference runs each layer's two edge GEMMs as one kernel (sphg_gnn_edge_layer)
        self.fused_edges = True
        # inference keeps the edge latent in bf16 only (no fp32 residual stream):
        # the 64 held-out scenes gave the same runout and free-surface errors
        # as with the fp32 stream (mean 0.20 / 0.14 dx, worst 0.85 / 0.39 dx)
        self.edge_bf16 = True
        # ... and gathers the sender latents into the edge layer's first GEMM
        # (sphg_gnn_edge_layer_nodes) instead of projecting them to P rows first
        self.edge_nodes = True

    # ------------------------------------------------------------ plumbing
    @property
    def stream(self) -> int:
        return self.torch.cuda.current_stream(self.device).cuda_stream

    def weights(self) -> dict:
        out = {k: v["w"].cpu().numpy().copy() for k, v in self.W.items()}
        out.update({k: v["w"].cpu().numpy().copy() for k, v in self.B.items()})
        return out

    def state(self) -> dict:
        d = self.weights()
        d["_vscale"] = np.array([self.vscale], np.float64)
        d["_x0"] = np.array([1 if self.use_x0 else 0], np.int32)
        d["_norm"] = self.norm.cpu().numpy()
        return d

    @classmethod
    def from_state(cls, d: dict, device="cuda"):
        net = cls({k: v for k, v in d.items() if not k.startswith("_")}, device=device)
        net.vscale = float(d["_vscale"][0])
        net.use_x0 = bool(int(np.asarray(d.get("_x0", [0]))[0]))
        net.norm.copy_(net.torch.from_numpy(np.asarray(d["_norm"], np.float32)))
        return net

    def _gemm(self, A, B, Cm, M, N, K, acc=0, split=1):
        self.launches += 1
        _call(self.L.sphg_gemm_bf16_tn(_ptr(A), _ptr(B), _ptr(Cm), M, N, K, acc, split, _ptr(self.err), self.stream),
              "sphg_gemm_bf16_tn")

    @staticmethod
    def _split(M, N, K):
        bn = 128 if N % 128 == 0 else 64 if N % 64 == 0 else 32 if N % 32 == 0 else 16
        tiles = (M // 128) * (N // bn)
        return max(1, min(K // 64 // 2, (2 * 148) // max(tiles, 1)))

    def _ws(self, X, Wm, rows, N, K, mode, relu=0, bias=None, z=None, h=None, P=None, src=None, dst=None, nedge=0):
        """Weight-stationary GEMM X [rows x K] . Wm[N x K]^T with a fused epilogue."""
        e = GemmEpi(mode, relu, _ptr(bias), _ptr(z), _ptr(h), _ptr(P), _ptr(src), _ptr(dst), nedge)
        self.launches += 1
        _call(self.L.sphg_gemm_bf16_ws(_ptr(X), _ptr(Wm), rows, N, K, C.addressof(e), _ptr(self.err), self.stream),
              "sphg_gemm_bf16_ws")

    def _k(self, fn, *args):
        self.launches += 1
        _call(getattr(self.L, fn)(*args), fn)

    def _wgrad(self, dY, X, name, rows):
        """W.g += dY^T X through two transposes and one split-K GEMM."""
        t = self.torch
        w = self.W[name]
        out, inn = w["rows"], w["cols"]
        tA = self.bufs.get("tA", (out, rows), t.bfloat16)
        tB = self.bufs.get("tB", (inn, rows), t.bfloat16)
        self._k("sphg_gnn_transpose", _ptr(dY), 1 if dY.dtype == t.float32 else 0, _ptr(tA), rows, out, self.stream)
        self._k("sphg_gnn_transpose", _ptr(X), 1 if X.dtype == t.float32 else 0, _ptr(tB), rows, inn, self.stream)
        self._gemm(tA, tB, w["g"], out, inn, rows, acc=1, split=self._split(out, inn, rows))

    def _bgrad(self, dY, bname, rows):
        self._k("sphg_gnn_colsum", _ptr(dY), rows, dY.shape[1], _ptr(self.B[bname]["g"]), self.stream)

    def _bf16(self, x, name):
        t = self.torch
        y = self.bufs.get(name, tuple(x.shape), t.bfloat16)
        self._k("sphg_gnn_f32_to_bf16", _ptr(x), _ptr(y), x.numel(), self.stream)
        return y

    # ------------------------------------------------------------- forward
    def forward(self, b: Batch, keep: bool):
        """Network output [n_pad, L] (columns 0, 1 = normalised acceleration).
        keep: store what the backward pass needs (pre-activations and the
        bf16 inputs of every layer); otherwise the buffers are reused layer to
        layer and the pre-activations are never written."""
        t, L, G = self.torch, L_WIDTH, self.bufs.get
        f32, bf = t.float32, t.bfloat16
        W, B = self.W, self.B
        Np, Ep = b.n_pad, b.E_pad
        s = self.stream
        tag = (lambda l: str(l)) if keep else (lambda l: "0")
        opt = (lambda name, shape: G(name, shape, f32)) if keep else (lambda name, shape: None)
        na = G("na", (Np, L), bf)
        self._ws(b.fn, W["enc_n.w1"]["wb"], Np, L, F_IN, EPI_BIAS_ACT, 1, B["enc_n.b1"]["w"], opt("nz", (Np, L)), na)
        hf = G("hf", (Np, L), f32)
        hb = G("hb" + tag(0), (Np, L), bf)
        self._ws(na, W["enc_n.w2"]["wb"], Np, L, L, EPI_BIAS_ACT, 0, B["enc_n.b2"]["w"], hf, hb)
        bf_edges = self.edge_bf16 and not keep and self.fused_edges   # edge latent kept in bf16 only
        ef = None if bf_edges else G("ef", (Ep, L), f32)
        eb = G("eb" + tag(0), (Ep, L), bf)
        if bf_edges and self.edge_nodes:   # both encoder GEMMs in one kernel, the hidden rows kept on the SM
            self.launches += 1
            _call(self.L.sphg_gnn_edge_encoder(_ptr(b.fe), _ptr(eb), Ep, _ptr(W["enc_e.w1"]["wb"]),
                                               _ptr(B["enc_e.b1"]["w"]), _ptr(W["enc_e.w2"]["wb"]),
                                               _ptr(B["enc_e.b2"]["w"]), _ptr(self.err), s),
                  "sphg_gnn_edge_encoder")
        else:
            ea = G("ea", (Ep, L), bf)
            self._ws(b.fe, W["enc_e.w1"]["wb"], Ep, L, F_IN, EPI_BIAS_ACT, 1, B["enc_e.b1"]["w"], opt("ez", (Ep, L)),
                     ea)
            self._ws(ea, W["enc_e.w2"]["wb"], Ep, L, L, EPI_BIAS_ACT, 0, B["enc_e.b2"]["w"], ef, eb)
        P = G("P", (Np, 2 * L), f32)
        agg = G("agg", (Np, L), f32)
        gather = bf_edges and self.edge_nodes
        Pd = G("Pd", (Np, L), f32) if gather else None
        for l in range(LAYERS):
            p = f"p{l}."
            if gather:   # receiver rows per node, then one kernel with the sender rows gathered into its first GEMM
                wsd = W[p + "wsd"]["wb"]
                self._ws(hb, wsd[L:], Np, L, L, EPI_STORE, z=Pd)
                self.launches += 1
                _call(self.L.sphg_gnn_edge_layer_nodes(_ptr(eb), _ptr(eb), _ptr(hb), _ptr(Pd), Np, _ptr(b.src),
                                                       _ptr(b.dst), b.E, Ep, _ptr(W[p + "we"]["wb"]), _ptr(wsd),
                                                       _ptr(B[p + "be"]["w"]), _ptr(W[p + "w2"]["wb"]),
                                                       _ptr(B[p + "b2"]["w"]), _ptr(self.err), s),
                      "sphg_gnn_edge_layer_nodes")
            elif keep or not self.fused_edges:
                self._ws(hb, W[p + "wsd"]["wb"], Np, 2 * L, L, EPI_STORE, z=P)
                a = G("a" + tag(l), (Ep, L), bf)
                self._ws(eb, W[p + "we"]["wb"], Ep, L, L, EPI_EDGE, 1, B[p + "be"]["w"], opt("z" + tag(l), (Ep, L)), a,
                         P, b.src, b.dst, b.E)
                eb = G("eb" + tag(l + 1), (Ep, L), bf)
                self._ws(a, W[p + "w2"]["wb"], Ep, L, L, EPI_RESID, 0, B[p + "b2"]["w"], ef, eb)   # e += relu(z) W2^T + b2
            else:   # both edge GEMMs in one kernel, the hidden rows never leave the SM; eb updated in place
                self._ws(hb, W[p + "wsd"]["wb"], Np, 2 * L, L, EPI_STORE, z=P)
                self.launches += 1
                _call(self.L.sphg_gnn_edge_layer(_ptr(eb), _ptr(ef), _ptr(eb), _ptr(P), _ptr(b.src), _ptr(b.dst),
                                                 b.E, Ep, _ptr(W[p + "we"]["wb"]), _ptr(B[p + "be"]["w"]),
                                                 _ptr(W[p + "w2"]["wb"]), _ptr(B[p + "b2"]["w"]), _ptr(self.err), s),
                      "sphg_gnn_edge_layer")
            cat = G("cat" + tag(l), (Np, 2 * L), bf)
            if bf_edges:   # the receiver sums straight into the node MLP's input rows
                self._k("sphg_gnn_segsum_cat", _ptr(eb), _ptr(b.off), _ptr(hb), _ptr(cat), b.n, Np, L, AGG_SCALE, s)
            else:
                self._k("sphg_gnn_segsum", _ptr(ef), _ptr(b.off), _ptr(agg), b.n, L, AGG_SCALE, s)
                self._k("sphg_gnn_node_concat", _ptr(hb), _ptr(agg), _ptr(cat), Np, L, s)
            hb = G("hb" + tag(l + 1), (Np, L), bf)
            if gather:   # both node GEMMs in one kernel, the hidden rows kept on the SM; h += relu(y) V2^T + c2
                self.launches += 1
                _call(self.L.sphg_gnn_node_mlp(_ptr(cat), Np, _ptr(W[p + "v1"]["wb"]), _ptr(B[p + "c1"]["w"]),
                                               _ptr(W[p + "v2"]["wb"]), _ptr(B[p + "c2"]["w"]), _ptr(hf), _ptr(hb),
                                               _ptr(self.err), s),
                      "sphg_gnn_node_mlp")
            else:
                ya = G("ya" + tag(l), (Np, L), bf)
                self._ws(cat, W[p + "v1"]["wb"], Np, L, 2 * L, EPI_BIAS_ACT, 1, B[p + "c1"]["w"],
                         opt("y" + tag(l), (Np, L)), ya)
                self._ws(ya, W[p + "v2"]["wb"], Np, L, L, EPI_RESID, 0, B[p + "c2"]["w"], hf, hb)  # h += relu(y) V2^T + c2
        dua = G("dua", (Np, L), bf)
        self._ws(hb, W["dec.w1"]["wb"], Np, L, L, EPI_BIAS_ACT, 1, B["dec.b1"]["w"], opt("du", (Np, L)), dua)
        out = G("out", (Np, L), f32)
        self._ws(dua, W["dec.w2"]["wb"], Np, L, L, EPI_BIAS_ACT, 0, B["dec.b2"]["w"], out, None)
        return out

    # ------------------------------------------------------------ backward
    def zero_grad(self):
        for d in list(self.W.values()) + list(self.B.values()):
            d["g"].zero_()

    def loss(self, b: Batch, out, delta: float = 0.0):
        """Masked mean squared error over the 2 acceleration columns (Huber
        beyond |d| = delta when delta > 0); returns d loss / d out."""
        t = self.torch
        dout = self.bufs.get("dout", (b.n_pad, L_WIDTH), t.float32)
        self.loss_buf.zero_()
        self._k("sphg_gnn_mse", _ptr(out), L_WIDTH, _ptr(b.target), NOUT, _ptr(b.mask), b.n_pad,
                1.0 / (NOUT * max(b.n_real, 1)), delta, _ptr(dout), _ptr(self.loss_buf), self.stream)
        return dout

    def snapshot(self):
        return {k: d["w"].clone() for k, d in list(self.W.items()) + list(self.B.items())}

    def restore(self, snap):
        """Master weights from a snapshot; the bf16 copies follow."""
        t = self.torch
        for k, d in list(self.W.items()) + list(self.B.items()):
            d["w"].copy_(snap[k])
        for d in self.W.values():
            d["wb"].copy_(d["w"].to(t.bfloat16))
            d["wt"].copy_(d["w"].t().to(t.bfloat16))

    def backward(self, b: Batch, dout, trace: dict | None = None):
        """Gradients into W[.]["g"] / B[.]["g"]; with a trace dict, copies of the
        incoming node and edge gradients of every layer (and of the encoders)
        are kept for a stage-by-stage check."""
        t, L, G = self.torch, L_WIDTH, self.bufs.get
        f32, bf = t.float32, t.bfloat16
        Np, Ep = b.n_pad, b.E_pad
        s = self.stream
        # decoder
        self._bgrad(dout, "dec.b2", Np)
        self._wgrad(dout, G("dua", (Np, L), bf), "dec.w2", Np)
        tmpN = G("tmpN", (Np, L), f32)
        self._ws(self._bf16(dout, "doutb"), self.W["dec.w2"]["wt"], Np, L, L, EPI_STORE, z=tmpN)
        dy = G("dy", (Np, L), f32)
        dyb = G("dyb", (Np, L), bf)
        self._k("sphg_gnn_relu_bwd", _ptr(tmpN), _ptr(G("du", (Np, L), f32)), _ptr(dy), _ptr(dyb), Np * L, s)
        self._bgrad(dy, "dec.b1", Np)
        self._wgrad(dy, G(f"hb{LAYERS}", (Np, L), bf), "dec.w1", Np)
        dh = G("dh", (Np, L), f32)
        self._ws(dyb, self.W["dec.w1"]["wt"], Np, L, L, EPI_STORE, z=dh)
        de = G("de", (Ep, L), f32, zero=True)
        dcat = G("dcat", (Np, 2 * L), f32)
        dagg = G("dagg", (Np, L), f32)
        da = G("da", (Ep, L), f32)
        dz = G("dz", (Ep, L), f32)
        dzb = G("dzb", (Ep, L), bf)
        dP = G("dP", (Np, 2 * L), f32)
        for l in reversed(range(LAYERS)):
            p = f"p{l}."
            if trace is not None:
                trace[l] = (dh.clone(), de.clone())
            hb, eb = G(f"hb{l}", (Np, L), bf), G(f"eb{l}", (Ep, L), bf)
            z, a = G(f"z{l}", (Ep, L), f32), G(f"a{l}", (Ep, L), bf)
            y, ya, cat = G(f"y{l}", (Np, L), f32), G(f"ya{l}", (Np, L), bf), G(f"cat{l}", (Np, 2 * L), bf)
            # node update h' = h + relu(y) V2^T + c2
            self._bgrad(dh, p + "c2", Np)
            self._wgrad(dh, ya, p + "v2", Np)
            self._ws(self._bf16(dh, "dhb"), self.W[p + "v2"]["wt"], Np, L, L, EPI_STORE, z=tmpN)
            self._k("sphg_gnn_relu_bwd", _ptr(tmpN), _ptr(y), _ptr(dy), _ptr(dyb), Np * L, s)
            self._bgrad(dy, p + "c1", Np)
            self._wgrad(dy, cat, p + "v1", Np)
            self._ws(dyb, self.W[p + "v1"]["wt"], Np, 2 * L, L, EPI_STORE, z=dcat)
            self._k("sphg_gnn_node_concat_bwd", _ptr(dcat), _ptr(dh), _ptr(dagg), b.n, L, s)
            self._k("sphg_gnn_segsum_bwd", _ptr(dagg), _ptr(b.dst), _ptr(de), b.E, L, AGG_SCALE, s)
            # edge update e' = e + relu(z) W2^T + b2
            self._bgrad(de, p + "b2", Ep)
            self._wgrad(de, a, p + "w2", Ep)
            self._ws(self._bf16(de, "deb"), self.W[p + "w2"]["wt"], Ep, L, L, EPI_STORE, z=da)
            self._k("sphg_gnn_relu_bwd", _ptr(da), _ptr(z), _ptr(dz), _ptr(dzb), Ep * L, s)
            self._bgrad(dz, p + "be", Ep)
            self._wgrad(dz, eb, p + "we", Ep)
            self._ws(dzb, self.W[p + "we"]["wt"], Ep, L, L, EPI_ACC, z=de)
            dP.zero_()
            self._k("sphg_gnn_gather_bwd", _ptr(dz), _ptr(b.src), _ptr(b.off), _ptr(dP), b.n, b.E, L, s)
            self._wgrad(dP, hb, p + "wsd", Np)
            self._ws(self._bf16(dP, "dPb"), self.W[p + "wsd"]["wt"], Np, L, 2 * L, EPI_ACC, z=dh)
        if trace is not None:
            trace["enc"] = (dh.clone(), de.clone())
        # encoders
        for side, d, rows, feat in (("n", dh, Np, b.fn), ("e", de, Ep, b.fe)):
            enc = "enc_" + side
            zbuf = G(side + "z", (rows, L), f32)
            abuf = G(side + "a", (rows, L), bf)
            tmp = G("tmp" + side, (rows, L), f32)
            self._bgrad(d, enc + ".b2", rows)
            self._wgrad(d, abuf, enc + ".w2", rows)
            self._ws(self._bf16(d, "d" + side + "b"), self.W[enc + ".w2"]["wt"], rows, L, L, EPI_STORE, z=tmp)
            dzz = G("dzz" + side, (rows, L), f32)
            dzzb = G("dzzb" + side, (rows, L), bf)
            self._k("sphg_gnn_relu_bwd", _ptr(tmp), _ptr(zbuf), _ptr(dzz), _ptr(dzzb), rows * L, s)
            self._bgrad(dzz, enc + ".b1", rows)
            self._wgrad(dzz, feat, enc + ".w1", rows)

    def adam(self, lr: float, b1=0.9, b2=0.999, eps=1e-8):
        self.adam_step += 1
        s = self.stream
        for d in self.W.values():
            self._k("sphg_gnn_adam", _ptr(d["w"]), _ptr(d["g"]), _ptr(d["m"]), _ptr(d["v"]), _ptr(d["wb"]),
                    _ptr(d["wt"]), d["rows"], d["cols"], lr, b1, b2, eps, self.adam_step, d["lim"], s)
        for d in self.B.values():
            self._k("sphg_gnn_adam", _ptr(d["w"]), _ptr(d["g"]), _ptr(d["m"]), _ptr(d["v"]), None, None,
                    d["rows"], 1, lr, b1, b2, eps, self.adam_step, d["lim"], s)

    def check_device_errors(self):
        if int(self.err.item()) != 0:
            raise SPHError(6, "tcgen05 GEMM wait timed out")

    # --------------------------------------------------------------- batch
    def make_batch(self, x, nodes, vhist, head: int, grid: Grid, inv2h: float, target=None, x0=None) -> Batch:
        """Graph, node and edge features of the particles x [n, 2] (f64,
        device) with velocity history vhist [5, n, 2] (f32) at ring slot head
        and reference positions x0 [n, 2] (f64; the displacement features
        stay zero for a network trained without them, or without x0)."""
        t = self.torch
        n = x.shape[0]
        off, src, dst, E = self.graph.build(x, n, grid, self.stream)
        Np, Ep = pad128(n), pad128(E)
        fn = self.bufs.get("fn", (Np, F_IN), t.bfloat16)
        fe = self.bufs.get("fe", (Ep, F_IN), t.bfloat16)
        ref = x0 if self.use_x0 else None
        self._k("sphg_gnn_node_features", _ptr(x), _ptr(ref), _ptr(vhist), head, _ptr(nodes), n, Np, inv2h,
                1.0 / self.vscale, _ptr(fn), self.stream)
        self._k("sphg_gnn_edge_features", _ptr(x), _ptr(ref), _ptr(nodes), _ptr(src), _ptr(dst), E, Ep,
                float(inv2h), _ptr(fe), self.stream)
        b = Batch(n, Np, E, Ep, x, nodes, off, src, dst, fn, fe)
        if target is not None:
            b.target = self.bufs.get("target", (Np, NOUT), t.float32)
            b.target[:n] = target
            b.mask = self.bufs.get("mask", (Np,), t.float32, zero=True)
            typ = nodes.view(t.int32)[:, 7]
            b.mask[:n] = (typ != GNN_BOUNDARY).to(t.float32)
            b.n_real = int((typ != GNN_BOUNDARY).sum().item())
        return b

    def train_step(self, b: Batch, lr: float, delta: float = 0.0) -> float:
        self.zero_grad()
        out = self.forward(b, keep=True)
        dout = self.loss(b, out, delta)
        self.backward(b, dout)
        self.adam(lr)
        return float(self.loss_buf.item())


# ---------------------------------------------------------------- rollouts

def node_table(scene, offset: float, dts: float, kind: str) -> np.ndarray:
    """Per-particle constants of one scene (all phases, in phase order)."""
    rows = []
    xl, xr, yf = scene.box
    p = scene.params
    porosity = p.soil.porosity if kind == "submerged" else 0.0
    phi = p.soil.phi if kind in ("dry", "submerged") else 0.0
    for P in scene.phases:
        a = np.zeros(P.n, NODE_DTYPE)
        a["xl"], a["xr"], a["yf"] = xl + offset, xr + offset, yf
        a["dts"], a["porosity"], a["phi"] = dts, porosity, phi
        a["mass"] = P.mass
        real = np.asarray(P.itype) > 0
        a["type"] = np.where(real, GNN_WATER if P.material == SPHG_WATER else GNN_SOIL, GNN_BOUNDARY)
        rows.append(a)
    return np.concatenate(rows)


@dataclass
class GroupRollout:
    """Positions every k steps of one ensemble group (all phases, phase order)."""
    kind: str
    nodes: np.ndarray            # NODE_DTYPE [n]
    X: object                    # [T, n, 2] f64 device
    scene_idx: list              # per member: int64 device index of its nodes
    members: list                # ensemble scene indices
    grid: Grid
    inv2h: float
    h: float
    dx: float
    plain_ms: float = 0.0        # device time of the plain solver per step
    boxes: list = field(default_factory=list)
    scene_idx_np: list = field(default_factory=list)
    x0: object = None            # [n, 2] f64 reference positions (the first snapshot)
    nodes_dev: object = None     # [n, 32] uint8
    typ_dev: object = None       # [n] int32
    dts_dev: object = None       # [n] f32

    def finish(self, torch, device):
        self.scene_idx_np = [i.cpu().numpy() for i in self.scene_idx]
        if self.x0 is None:
            self.x0 = self.X[0]
        self.nodes_dev = torch.from_numpy(self.nodes.view(np.uint8).reshape(-1, 32).copy()).to(device)
        self.typ_dev = torch.from_numpy(self.nodes["type"].copy()).to(device)
        self.dts_dev = torch.from_numpy(self.nodes["dts"].copy()).to(device)
        return self


def _group_grid(g, radius: float) -> Grid:
    p = g.scene.params
    xmin, ymin = p.x_min - 4 * radius, p.y_min - 4 * radius
    nx = int(math.ceil((p.x_max + 4 * radius - xmin) / radius)) + 1
    ny = int(math.ceil((p.y_max + 4 * radius - ymin) / radius)) + 1
    return Grid(xmin, ymin, radius, nx, ny)


def _group_nodes(ens, g):
    parts = [[] for _ in g.scene.phases]
    for local, m in enumerate(g.members):
        sc = ens.built[m]
        dts = K_STRIDE * g.rows[local][0]
        tab = node_table(sc, g.offsets[local], dts, g.kind)
        a = 0
        for k, P in enumerate(sc.phases):
            parts[k].append(tab[a:a + P.n])
            a += P.n
    return np.concatenate([np.concatenate(p) for p in parts])


def _scene_index(g, torch, device):
    idx = []
    base = np.cumsum([0] + [P.n for P in g.scene.phases])
    for local in range(len(g.members)):
        parts = [np.arange(base[k] + a, base[k] + b) for k, (a, b) in
                 ((k, g.ranges[k][local]) for k in range(len(g.scene.phases)))]
        idx.append(torch.from_numpy(np.concatenate(parts).astype(np.int64)).to(device))
    return idx


def rollout_ensemble(ens, strides: int, device="cuda"):
    """Run every group of an Ensemble for `strides` strides of k steps and
    keep the positions (f64) of every particle after each stride (T =
    strides + 1 snapshots, the first the initial state)."""
    torch = _torch()
    dev = torch.device(device)
    stream = torch.cuda.current_stream(dev).cuda_stream
    ens.set_stream(stream)
    out = []
    for g, sv in zip(ens.groups, ens.solvers):
        n_ph = [P.n for P in g.scene.phases]
        n = sum(n_ph)
        X = torch.empty((strides + 1, n, 2), dtype=torch.float64, device=dev)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        steps_ms = 0.0
        for t in range(strides + 1):
            if t:
                ev0.record()
                sv.time_integration(K_STRIDE)
                ev1.record()
                ev1.synchronize()
                steps_ms += ev0.elapsed_time(ev1)
            a = 0
            for k, nk in enumerate(n_ph):
                sv.export_xv(k + 1, X[t, a:a + nk].data_ptr(), None)
                a += nk
        h = float(g.scene.phases[0].hsml[0])
        dx = float(g.scene.phases[0].dspp)
        r = GroupRollout(g.kind, _group_nodes(ens, g), X, _scene_index(g, torch, dev), list(g.members),
                         _group_grid(g, 2.0 * h), 1.0 / (2.0 * h), h, dx,
                         steps_ms / max(strides * K_STRIDE, 1))
        r.boxes = [ens.built[m].box for m in g.members]
        out.append(r.finish(torch, dev))
    torch.cuda.synchronize(dev)
    return out


def fd_velocity(r: GroupRollout, t: int, idx=None):
    """Stride velocity (x_t - x_{t-1}) / D of the nodes idx (all when None), f32."""
    if idx is None:
        d = r.X[t] - r.X[t - 1]
        return (d / r.dts_dev.double()[:, None]).float()
    d = r.X[t].index_select(0, idx) - r.X[t - 1].index_select(0, idx)
    return (d / r.dts_dev.index_select(0, idx).double()[:, None]).float()


def fd_acceleration(r: GroupRollout, t: int, idx):
    """Stride acceleration (x_{t+1} - 2 x_t + x_{t-1}) / D^2 of the nodes idx (f64)."""
    x0, x1, x2 = (r.X[t + j].index_select(0, idx) for j in (-1, 0, 1))
    dts = r.dts_dev.index_select(0, idx).double()[:, None]
    return (x2 - 2.0 * x1 + x0) / (dts * dts)


def scene_rollout(solver, scene, kind: str, strides: int, device="cuda", x0=None) -> GroupRollout:
    """Positions of one running single-scene Solver now and after each of
    `strides` further strides of k steps (T = strides + 1 snapshots).  The
    reference positions are x0 when given (e.g. the scene's initial
    lattice), else the first snapshot."""
    torch = _torch()
    dev = torch.device(device)
    solver.set_stream(torch.cuda.current_stream(dev).cuda_stream)
    sizes = [P.n for P in scene.phases]
    n = sum(sizes)
    X = torch.empty((strides + 1, n, 2), dtype=torch.float64, device=dev)
    for t in range(strides + 1):
        if t:
            solver.time_integration(K_STRIDE)
        a = 0
        for k, nk in enumerate(sizes):
            solver.export_xv(k + 1, X[t, a:a + nk].data_ptr(), None)
            a += nk
    h = float(scene.phases[0].hsml[0])
    p = scene.params
    radius = 2.0 * h
    xmin, ymin = p.x_min - 4 * radius, p.y_min - 4 * radius
    grid = Grid(xmin, ymin, radius, int(math.ceil((p.x_max + 4 * radius - xmin) / radius)) + 1,
                int(math.ceil((p.y_max + 4 * radius - ymin) / radius)) + 1)
    nodes = node_table(scene, 0.0, K_STRIDE * p.dt, kind)
    r = GroupRollout(kind, nodes, X, [torch.arange(n, device=dev)], [0], grid, 1.0 / radius, h,
                     float(scene.phases[0].dspp))
    r.boxes = [scene.box]
    if x0 is not None:
        r.x0 = x0
    torch.cuda.synchronize(dev)
    return r.finish(torch, dev)


def normalisation(rollouts, t0: int = HIST, snapshots: int = 24, nodes: int = 100_000, seed: int = 0):
    """Velocity scale and per-component acceleration mean / std over real
    particles of the training rollouts (stride finite differences), from up
    to `snapshots` evenly spaced snapshots and `nodes` random real particles
    of each group."""
    torch = _torch()
    g = torch.Generator(device=rollouts[0].X.device)
    g.manual_seed(seed)
    vs, acc = [], []
    for r in rollouts:
        real = torch.nonzero(r.typ_dev != GNN_BOUNDARY).flatten()
        if real.numel() > nodes:
            real = real[torch.randperm(real.numel(), device=real.device, generator=g)[:nodes]]
        T = r.X.shape[0]
        for t in range(t0, T - 1, max(1, (T - 1 - t0) // snapshots)):
            vs.append(fd_velocity(r, t, real).double())
            acc.append(fd_acceleration(r, t, real))
    v = torch.cat(vs)
    a = torch.cat(acc)
    vscale = float(v.std().item()) or 1.0
    return vscale, [float(a[:, 0].mean()), float(a[:, 1].mean()), float(a[:, 0].std()) or 1.0,
                    float(a[:, 1].std()) or 1.0]


def sample_batch(net: MPNet, r: GroupRollout, t: int, members: list, noise: float, gen=None) -> Batch:
    """Training batch: the chosen member scenes of a group at snapshot t
    (HIST <= t < T - 1); input velocities carry Gaussian noise of std
    noise * vscale (the target is taken relative to the noisy current
    velocity, so the network learns to correct it)."""
    torch = net.torch
    idx = torch.cat([r.scene_idx[m] for m in members])
    x = r.X[t].index_select(0, idx).contiguous()
    vh = torch.stack([fd_velocity(r, t - j, idx) for j in range(HIST)]).contiguous()
    nodes = r.nodes_dev.index_select(0, idx).contiguous()
    typ = r.typ_dev.index_select(0, idx)
    dts = r.dts_dev.index_select(0, idx)
    acc = fd_acceleration(r, t, idx).float()
    if noise > 0:
        nz = torch.randn(vh.shape, device=x.device, generator=gen) * (noise * net.vscale)
        nz[:, typ == GNN_BOUNDARY] = 0
        vh = vh + nz
        acc = acc - nz[0] / dts[:, None]
    nrm = net.norm
    # heavy tails (wall impacts, splashes) are clamped at 20 std
    target = ((acc - nrm[:2]) / nrm[2:]).clamp_(-TARGET_CLAMP, TARGET_CLAMP)
    return net.make_batch(x, nodes, vh, 0, r.grid, r.inv2h, target=target,
                          x0=r.x0.index_select(0, idx).contiguous())


def train(net: MPNet, rollouts, iters: int, lr0=3e-4, lr1=3e-5, batch_nodes=120_000, noise=0.002, seed=0,
          log_every=0, delta=HUBER_DELTA, balance=False, kind_weight=None):
    """Adam on random (group, snapshot, member subset) batches with a Huber
    loss; the learning rate decays exponentially from lr0 to lr1.  The
    weights with the lowest running loss (exponential average over ~50
    iterations, checked every 50) are kept.  Returns the loss history."""
    torch = net.torch
    rng = np.random.Generator(np.random.PCG64(seed))
    gen = torch.Generator(device=net.device)
    gen.manual_seed(seed)
    # groups drawn by particle count, or each kind (group) equally often
    sizes = np.array([1.0 if balance else sum(int(r.scene_idx[m].numel()) for m in range(len(r.members)))
                      for r in rollouts], float)
    if kind_weight:
        sizes *= np.array([kind_weight.get(r.kind, 1.0) for r in rollouts])
    losses = []
    ema, best, best_w = None, math.inf, None
    for it in range(iters):
        r = rollouts[rng.choice(len(rollouts), p=sizes / sizes.sum())]
        T = r.X.shape[0]
        t = int(rng.integers(HIST, T - 1))
        order = rng.permutation(len(r.members))
        chosen, total = [], 0
        for m in order:
            k = int(r.scene_idx[m].numel())
            if chosen and total + k > batch_nodes:
                continue
            chosen.append(int(m))
            total += k
        b = sample_batch(net, r, t, chosen, noise, gen)
        lr = lr0 * (lr1 / lr0) ** (it / max(iters - 1, 1))
        losses.append(net.train_step(b, lr, delta))
        ema = losses[-1] if ema is None else 0.98 * ema + 0.02 * losses[-1]
        if it >= 100 and it % 50 == 0 and ema < best:
            best, best_w = ema, net.snapshot()
        if log_every and it % log_every == 0:
            print(f"iter {it} loss {losses[-1]:.4f} ema {ema:.4f} nodes {b.n} edges {b.E}", flush=True)
    if best_w is not None and ema > best:
        net.restore(best_w)
    net.check_device_errors()
    return losses


# ------------------------------------------------------------ the stepper

class LearnedStepper:
    """Learned strides over one group's particles, starting from snapshot
    t0 of a rollout (positions and the HIST stride velocities up to t0).
    mode 'net' uses the network, 'gravity' the stepper with a = g (the
    method without the network), both with the same stride update and walls.

    With a solver (holding the same group at snapshot t0, phase sizes in
    phase_sizes) the fallback gates are live: a stride that fails them is
    discarded and the solver, which stays authoritative, advances from the
    last state it holds to the end of that stride; the learned strides then
    continue from its positions and stride velocities.  The solver never
    receives learned positions, so its density and stress fields stay its
    own."""

    def __init__(self, net: MPNet, r: GroupRollout, t0: int = HIST, mode: str = "net", solver=None,
                 phase_sizes=None):
        torch = net.torch
        self.net, self.r, self.mode = net, r, mode
        dev = net.device
        self.n = r.X.shape[1]
        self.x = r.X[t0].clone()
        self.vh = torch.stack([fd_velocity(r, t0 - j) for j in range(HIST)]).contiguous()
        self.head = 0
        self.nodes = r.nodes_dev
        self.solver, self.phase_sizes = solver, phase_sizes
        # the solver's own trajectory at stride boundaries (oldest first)
        self.solver_x = [r.X[t0 - j].clone() for j in range(HIST, -1, -1)] if solver is not None else None
        self.synced = 0            # learned strides done when the solver was last at the same time
        self.sig = [torch.zeros(self.n, dtype=torch.float64, device=dev) for _ in range(2)]
        self.gate = torch.zeros(4, dtype=torch.float64, device=dev)
        typ = r.nodes["type"]
        self.e_floor = float((r.nodes["mass"][typ != GNN_BOUNDARY].astype(np.float64) * (-GRAVITY) * r.dx).sum())
        self.fallbacks = 0
        self.strides = 0
        self.batch = None
        self._graph()
        self._density(self.sig[0])
        self.energy, self.energy_ke = self._energy(self.sig[0])

    def _energy(self, sig_new):
        """(kinetic + potential, kinetic) energy of the current state; the
        density sums of the gate against sig[0] land in self.gate."""
        net = self.net
        _call(net.L.sphg_gnn_gate_sums(_ptr(sig_new), _ptr(self.sig[0]), _ptr(self.x), _ptr(self.vh[self.head]),
                                       _ptr(self.nodes), self.n, -GRAVITY, _ptr(self.gate), net.stream),
              "sphg_gnn_gate_sums")
        g = self.gate.cpu().numpy()
        self.last_gate = g
        return float(g[2] + g[3]), float(g[2])

    def _graph(self):
        self.batch = self.net.make_batch(self.x, self.nodes, self.vh, self.head, self.r.grid, self.r.inv2h,
                                         x0=self.r.x0)

    def _density(self, out):
        b = self.batch
        _call(self.net.L.sphg_gnn_number_density(_ptr(self.x), _ptr(b.off), _ptr(b.src), self.n, self.r.h,
                                                 _ptr(out), self.net.stream), "sphg_gnn_number_density")

    def _pred(self):
        net, torch = self.net, self.net.torch
        if self.mode == "net":
            return net.forward(self.batch, keep=False)
        out = net.bufs.get("gravity_pred", (self.batch.n_pad, L_WIDTH), torch.float32, zero=True)
        out[:, 1] = (GRAVITY - float(net.norm[1])) / float(net.norm[3])
        out[:, 0] = -float(net.norm[0]) / float(net.norm[2])
        return out

    def step(self):
        """One stride: network, update, gates; a failed stride is replaced
        by the solver's.  Returns True when the learned stride was kept."""
        net = self.net
        pred = self._pred()
        new = (self.head + HIST - 1) % HIST
        _call(net.L.sphg_gnn_stride_update(_ptr(pred), L_WIDTH, _ptr(net.norm), _ptr(self.nodes), _ptr(self.x),
                                           _ptr(self.vh), self.head, new, self.n, 1e-9, net.stream),
              "sphg_gnn_stride_update")
        self.head = new
        self._graph()
        self._density(self.sig[1])
        energy, ke = self._energy(self.sig[1])
        g = self.last_gate
        rms = math.sqrt(g[0] / max(g[1], 1.0))
        rise = (energy - self.energy) / (max(self.energy_ke, 0.0) + self.e_floor)
        self.last_rms, self.last_rise = rms, rise
        failed = self.solver is not None and (not math.isfinite(rms) or rms > GATE_DENSITY or rise > GATE_ENERGY)
        if failed:
            self.fallbacks += 1
            self._catch_up(self.strides + 1)
            self._graph()
            self._density(self.sig[1])
            energy, ke = self._energy(self.sig[1])
        self.energy, self.energy_ke = energy, ke
        self.sig.reverse()
        self.strides += 1
        return not failed

    def _catch_up(self, upto: int):
        """The solver advances from the last time it holds to `upto` strides
        after t0; positions and stride velocities are taken from it."""
        torch = self.net.torch
        for _ in range(upto - self.synced):
            self.solver.time_integration(K_STRIDE)
            x = torch.empty_like(self.x)
            a = 0
            for k, nk in enumerate(self.phase_sizes):
                self.solver.export_xv(k + 1, x[a:a + nk].data_ptr(), None)
                a += nk
            self.solver_x.append(x)
            self.solver_x.pop(0)
        self.synced = upto
        self.x.copy_(self.solver_x[-1])
        dts = self.r.dts_dev.double()[:, None]
        for j in range(HIST):
            self.vh[j].copy_(((self.solver_x[-1 - j] - self.solver_x[-2 - j]) / dts).float())
        self.head = 0


# -------------------------------------------------------------- evaluation

def front_and_surface(x, typ, material, box, dx, bin_w=None):
    """Runout (furthest x of the column material from the left wall) and the
    free-surface profile (highest y per x bin of width 2 dx, -inf where empty)."""
    p = x[typ == material]
    if p.size == 0:
        return 0.0, np.full(0, -np.inf)
    bin_w = bin_w or 2.0 * dx
    runout = float(p[:, 0].max() - box[0])
    bins = np.clip(np.floor((p[:, 0] - box[0]) / bin_w).astype(np.int64), 0, None)
    prof = np.full(int(bins.max()) + 1, -np.inf)
    np.maximum.at(prof, bins, p[:, 1])
    return runout, prof


def scene_errors(x_pred, x_ref, nodes, kind, box, dx):
    """Runout and mean free-surface errors in units of dx."""
    typ = nodes["type"]
    mat = GNN_WATER if kind == "dam_break" else GNN_SOIL
    r_p, s_p = front_and_surface(x_pred, typ, mat, box, dx)
    r_r, s_r = front_and_surface(x_ref, typ, mat, box, dx)
    m = min(s_p.size, s_r.size)
    both = np.isfinite(s_p[:m]) & np.isfinite(s_r[:m])
    surf = float(np.abs(s_p[:m][both] - s_r[:m][both]).mean() / dx) if both.any() else float("nan")
    return abs(r_p - r_r) / dx, surf


def evaluate(net: MPNet, rollouts, t0: int = HIST, strides: int | None = None, mode="net", solvers=None):
    """Roll every group out from snapshot t0 for `strides` learned strides and
    compare each scene with the plain solver's snapshot at the same time.
    Returns per-scene errors, timing and fallback counts."""
    torch = net.torch
    rows = []
    wall = 0.0
    psteps = 0
    plain_ms = 0.0
    fallbacks = 0
    for gi, r in enumerate(rollouts):
        T = r.X.shape[0]
        ns = strides if strides is not None else T - 1 - t0
        solver, sizes = (solvers[gi] if solvers else (None, None))
        st = LearnedStepper(net, r, t0, mode, solver, sizes)
        torch.cuda.synchronize(net.device)
        c0 = time.perf_counter()
        for _ in range(ns):
            st.step()
        torch.cuda.synchronize(net.device)
        wall += time.perf_counter() - c0
        psteps += r.X.shape[1] * ns * K_STRIDE
        plain_ms += r.plain_ms * ns * K_STRIDE
        fallbacks += st.fallbacks
        xp = st.x.cpu().numpy()
        xr = r.X[t0 + ns].cpu().numpy()
        for local, m in enumerate(r.members):
            idx = r.scene_idx_np[local]
            ro, sf = scene_errors(xp[idx], xr[idx], r.nodes[idx], r.kind, r.boxes[local], r.dx)
            rows.append(dict(scene=m, kind=r.kind, n=int(idx.size), runout_dx=ro, surface_dx=sf))
    return dict(scenes=rows, learned_particle_steps_per_s=psteps / max(wall, 1e-12),
                plain_particle_steps_per_s=psteps / max(plain_ms * 1e-3, 1e-12), fallbacks=fallbacks,
                wall_s=wall)


# ------------------------------------------------------------ experiment

def held_out(seed: int) -> bool:
    """The 20 % of seeds held out of training: first byte of the SHA-256 of
    the seed's decimal text, modulo 5, equal to 0."""
    import hashlib
    return hashlib.sha256(str(seed).encode()).digest()[0] % 5 == 0


def split_specs(n_train_pool: int, n_test: int, test_min: int = 10_000, test_max: int = 60_000,
                dx: float = 0.004):
    """Training specs: the non-held-out seeds among the first n_train_pool.
    Test specs: the first n_test held-out seeds whose scene holds test_min to
    test_max particles (virtual particles included)."""
    from . import ensemble
    train = [s for s in ensemble.specs(n_train_pool) if not held_out(s.seed)]
    test, seed = [], 0
    while len(test) < n_test and seed < 100_000:
        if held_out(seed):
            sp = ensemble.spec(seed)
            n = ensemble.build_scene(sp, dx=dx).n_particles
            if test_min <= n <= test_max:
                test.append(sp)
        seed += 1
    return train, test


def _fallback_solvers(ens, strides0: int):
    """The held-out ensemble's own solvers advanced to the learned start."""
    torch = _torch()
    ens.set_stream(torch.cuda.current_stream().cuda_stream)
    ens.time_integration(strides0 * K_STRIDE)
    return [(sv, [P.n for P in g.scene.phases]) for g, sv in zip(ens.groups, ens.solvers)]


def summarise(res: dict) -> dict:
    sc = res["scenes"]
    ro = np.array([r["runout_dx"] for r in sc])
    sf = np.array([r["surface_dx"] for r in sc])
    kinds = {}
    for kind in sorted({r["kind"] for r in sc}):
        k_ro = np.array([r["runout_dx"] for r in sc if r["kind"] == kind])
        k_sf = np.array([r["surface_dx"] for r in sc if r["kind"] == kind])
        kinds[kind] = dict(scenes=int(k_ro.size), runout_dx_mean=float(np.nanmean(k_ro)),
                           runout_dx_median=float(np.nanmedian(k_ro)), surface_dx_mean=float(np.nanmean(k_sf)),
                           surface_dx_median=float(np.nanmedian(k_sf)),
                           within_1dx=float(np.mean((k_ro <= 1.0) & (k_sf <= 1.0))))
    return dict(scenes=len(sc), runout_dx_mean=float(np.nanmean(ro)), runout_dx_median=float(np.nanmedian(ro)),
                runout_dx_max=float(np.nanmax(ro)), surface_dx_mean=float(np.nanmean(sf)),
                surface_dx_median=float(np.nanmedian(sf)), surface_dx_max=float(np.nanmax(sf)),
                within_1dx=float(np.mean((ro <= 1.0) & (sf <= 1.0))), by_kind=kinds,
                learned_particle_steps_per_s=res["learned_particle_steps_per_s"],
                plain_particle_steps_per_s=res["plain_particle_steps_per_s"],
                speed_vs_plain=res["learned_particle_steps_per_s"] / res["plain_particle_steps_per_s"],
                fallbacks=res["fallbacks"])


def stride_bench(n_scenes: int, strides: int, weights=None, edge_bf16: bool = True, edge_nodes: bool = True):
    """Learned strides on the largest group of n_scenes held-out scenes (a
    history of HIST strides from the plain solver first): wall time per
    stride, forward time (CUDA events) and the graph size, as one JSON line."""
    import json
    from . import ensemble
    torch = _torch()
    _, specs = split_specs(0, n_scenes)
    ens = ensemble.Ensemble(specs, tune=False)
    roll = rollout_ensemble(ens, HIST)
    ens.close()
    path = weights or (DEFAULT_WEIGHTS if os.path.exists(DEFAULT_WEIGHTS) else None)
    net = MPNet.from_state(dict(np.load(path))) if path else MPNet(seed=0)
    net.edge_bf16 = edge_bf16
    net.edge_nodes = edge_nodes
    r = max(roll, key=lambda q: q.X.shape[1])
    LearnedStepper(net, r, HIST, "net").step()
    st = LearnedStepper(net, r, HIST, "net")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(strides):
        st.step()
    torch.cuda.synchronize()
    wall = (time.perf_counter() - t0) / strides
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(strides):
        net.forward(st.batch, keep=False)
    e1.record()
    e1.synchronize()
    n = r.X.shape[1]
    print(json.dumps(dict(nodes=n, edges=int(st.batch.E), kind=r.kind, strides=strides, ms_per_stride=wall * 1e3,
                          forward_ms=e0.elapsed_time(e1) / strides,
                          particle_steps_per_s=n * K_STRIDE / wall, weights=path or "random",
                          edge_bf16=edge_bf16, edge_nodes=edge_nodes)))


def main(argv=None):
    import argparse
    import json
    from . import ensemble
    ap = argparse.ArgumentParser(description="train and evaluate the learned particle stepper")
    ap.add_argument("--pool", type=int, default=256, help="seeds 0..pool-1, 80 %% of them for training")
    ap.add_argument("--test", type=int, default=64, help="held-out scenes of 10k-60k particles")
    ap.add_argument("--steps", type=int, default=2000, help="solver steps of every rollout")
    ap.add_argument("--iters", type=int, default=3000)
    ap.add_argument("--batch-nodes", type=int, default=120_000)
    ap.add_argument("--lr", type=float, nargs=2, default=(3e-4, 2e-5))
    ap.add_argument("--noise", type=float, default=0.002)
    ap.add_argument("--balance", action="store_true", help="draw each scene kind equally often")
    ap.add_argument("--kind-weight", nargs=2, action="append", metavar=("KIND", "W"), default=[],
                    help="multiply the draw probability of a scene kind (repeatable)")
    ap.add_argument("--weights", default=None, help="write the trained weights (.npz)")
    ap.add_argument("--load", default=None, help="evaluate these weights instead of training")
    ap.add_argument("--report", default=None, help="write the JSON report")
    ap.add_argument("--edge-fp32", action="store_true",
                    help="inference keeps the fp32 residual stream of the edge latent (default: bf16 only)")
    ap.add_argument("--edge-proj", action="store_true",
                    help="inference adds projected node rows (P) in the edge layer's epilogue instead of "
                         "gathering the node latents into its first GEMM")
    ap.add_argument("--stride-bench", type=int, default=0, metavar="S",
                    help="only time S learned strides on the first --test held-out scenes (no training)")
    a = ap.parse_args(argv)
    torch = _torch()
    if a.stride_bench:
        return stride_bench(a.test, a.stride_bench, a.load, not a.edge_fp32, not a.edge_proj)
    strides = a.steps // K_STRIDE
    train_specs, test_specs = split_specs(a.pool, a.test)
    report = dict(config=dict(pool=a.pool, train_scenes=len(train_specs), test_scenes=len(test_specs),
                              steps=a.steps, stride=K_STRIDE, iters=a.iters, batch_nodes=a.batch_nodes,
                              lr=list(a.lr), noise=a.noise, balance=a.balance, kind_weight=a.kind_weight,
                              edge_bf16=not a.edge_fp32, edge_nodes=not a.edge_proj,
                              width=L_WIDTH, layers=LAYERS))
    t0 = time.perf_counter()
    if a.load:
        net = MPNet.from_state(dict(np.load(a.load)))
    else:
        ens = ensemble.Ensemble(train_specs, tune=False)
        report["train_particles"] = ens.n_particles
        roll = rollout_ensemble(ens, strides)
        ens.close()
        report["rollout_s"] = time.perf_counter() - t0
        net = MPNet(seed=0)
        net.vscale, nrm = normalisation(roll)
        net.norm.copy_(torch.tensor(nrm))
        t1 = time.perf_counter()
        losses = train(net, roll, a.iters, a.lr[0], a.lr[1], a.batch_nodes, a.noise, log_every=250,
                       balance=a.balance, kind_weight={k: float(w) for k, w in a.kind_weight})
        torch.cuda.synchronize()
        report["train_s"] = time.perf_counter() - t1
        report["loss_first_100"] = float(np.mean(losses[:100]))
        report["loss_last_100"] = float(np.mean(losses[-100:]))
        del roll
        if a.weights:
            np.savez_compressed(a.weights, **net.state())
    net.edge_bf16 = not a.edge_fp32
    net.edge_nodes = not a.edge_proj
    torch.cuda.empty_cache()
    ens_t = ensemble.Ensemble(test_specs, tune=False)
    report["test_particles"] = ens_t.n_particles
    held = rollout_ensemble(ens_t, strides)
    ens_t.close()
    ens_f = ensemble.Ensemble(test_specs, tune=False)
    solvers = _fallback_solvers(ens_f, HIST)
    res_net = evaluate(net, held, HIST, mode="net", solvers=solvers)
    res_free = evaluate(net, held, HIST, mode="net")   # the same rollout with the fallback gates off
    res_grav = evaluate(net, held, HIST, mode="gravity")
    ens_f.close()
    report["learned"] = summarise(res_net)
    report["learned_gates_off"] = summarise(res_free)
    report["gravity_only"] = summarise(res_grav)
    report["per_scene"] = [dict(r, gates_off_runout_dx=f["runout_dx"], gates_off_surface_dx=f["surface_dx"],
                                gravity_runout_dx=g["runout_dx"], gravity_surface_dx=g["surface_dx"])
                           for r, f, g in zip(res_net["scenes"], res_free["scenes"], res_grav["scenes"])]
    report["total_s"] = time.perf_counter() - t0
    txt = json.dumps(report, indent=1)
    if a.report:
        with open(a.report, "w") as f:
            f.write(txt)
    print(json.dumps({k: v for k, v in report.items() if k != "per_scene"}, indent=1))


if __name__ == "__main__":
    main()
