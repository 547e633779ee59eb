"""Learned surrogate of the MOSFET current/charge map: an MLP trained and run on the tensor cores.

Network (one per device type): 5 inputs (Vgs, Vds, Vbs, log W, log L; each scaled to about
[-1, 1]) -> 4 hidden layers of 128 SiLU units -> 10 outputs, the drain current Id, the gate,
drain and bulk charges Qg, Qd, Qb, and the bias derivatives gm = dId/dVgs, gds = dId/dVds,
gmb = dId/dVbs, Cgg = dQg/dVgs, Cgd = dQg/dVds, Cgb = dQg/dVbs. Outputs are learned in a
compressed scale, y = asinh(x / s) per output, so that relative accuracy holds across the many
decades a MOSFET current spans.

Weights of the 128-wide layers are BF16 for the matrix products (FP32 master copies and Adam
moments), accumulation is FP32; those products run in ``xd_gemm_bf16`` (tcgen05 tensor cores,
include/xyce_surrogate.h) with the bias / SiLU / SiLU-derivative work fused into the epilogue. The
first layer (5 -> 128, 0.5% of the FLOPs) runs in FP32 on the CUDA cores so that the bias inputs
keep full precision (BF16 would round 1 V to ~4 mV, a 10% step of a subthreshold current). The
loss gradient, bias gradients, split-K reductions and the Adam update are the library's own
kernels as well. torch only owns the
buffers and orders the calls on a stream.

Shapes are padded for the tensor cores: inputs to 16 columns (K of the first layer), outputs to 16
(N of the last), the batch to a multiple of 128.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np

from . import _native

N_IN, N_HID, N_LAYERS, N_OUT = 5, 128, 4, 10
PAD_IN, PAD_OUT = 16, 16
OUTPUT_NAMES = ("Id", "Qg", "Qd", "Qb", "gm", "gds", "gmb", "Cgg", "Cgd", "Cgb")
# Scale of each output inside asinh(x / s). Near the operating magnitudes rather than at the
# smallest values: with a tiny scale the encoded value swings by ~20 within millivolts of a sign
# change (Id at Vds = 0, the charges), a near-discontinuity the network cannot fit.
OUTPUT_SCALE = np.array([1e-6, 1e-16, 1e-16, 1e-16, 1e-6, 1e-6, 1e-6, 1e-16, 1e-16, 1e-16])
VMAX = 1.2
LOG_W = (math.log(0.1e-6), math.log(10e-6))
LOG_L = (math.log(30e-9), math.log(500e-9))


def features(vgs, vds, vbs, w, l):
    """Scaled network inputs [n, 5] from biases (V) and geometry (m)."""
    def sc(x, lo, hi):
        return (2.0 * (x - lo) / (hi - lo)) - 1.0
    return np.stack([np.asarray(vgs) / VMAX, np.asarray(vds) / VMAX, np.asarray(vbs) / VMAX,
                     sc(np.log(w), *LOG_W), sc(np.log(l), *LOG_L)], 1)


# Encoded targets are clipped to +-ENC_CLIP: beyond it (|Id| > ~0.24 A, reached only by
# forward-biased junctions deep in the sampling box) the exact value is of no use to a warm start,
# and unclipped exponential tails would dominate the squared error.
ENC_CLIP = 20.0


def encode_targets(y):
    return np.clip(np.arcsinh(np.asarray(y) / OUTPUT_SCALE), -ENC_CLIP, ENC_CLIP)


def decode_outputs(z):
    return np.sinh(np.asarray(z)) * OUTPUT_SCALE


def _p(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


class _Lib:
    def __init__(self, torch, device):
        self.lib = _native.load()
        self.torch = torch
        self.dev = device
        self.err = torch.zeros(1, dtype=torch.int32, device=device)

    def stream(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream(self.dev).cuda_stream)

    def gemm(self, A, B, M, N, K, lda, ldb, epilogue, tile_n, *, C32=None, ldc=0, bias=None, Z=None, H=None, HT=None,
             ldt=0, Zin=None, splits=1):
        g = _native.XdGemmArgs()
        g.A, g.B = A.data_ptr(), B.data_ptr()
        g.M, g.N, g.K, g.lda, g.ldb, g.ldc, g.ldt = M, N, K, lda, ldb, ldc, ldt
        g.tile_n, g.epilogue = tile_n, epilogue
        for name, t in (("C32", C32), ("bias", bias), ("Z", Z), ("H", H), ("HT", HT), ("Zin", Zin)):
            setattr(g, name, None if t is None else t.data_ptr())
        g.err = self.err.data_ptr()
        rc = self.lib.xd_gemm_bf16(ctypes.byref(g), int(splits), self.stream())
        if rc < 0:
            _native.check(rc, "xd_gemm_bf16")
        return rc

    def check_err(self):
        if int(self.err.item()) != 0:
            raise _native.NativeError("a tensor-core kernel's internal wait expired")


EPI_F32, EPI_BIAS_F32, EPI_BIAS_SILU, EPI_SILU_BACK = 0, 1, 2, 3


@dataclass
class AdamConfig:
    lr: float = 2e-3
    beta1: float = 0.9
    beta2: float = 0.999
    eps: float = 1e-8


class SurrogateMLP:
    """One 5 -> 128^4 -> 10 SiLU network on a CUDA device, trained with the library's kernels."""

    def __init__(self, device=0, seed=0, max_batch=65536):
        import torch

        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.k = _Lib(torch, self.dev)
        g = torch.Generator().manual_seed(seed)
        dims = [(N_HID, N_IN)] + [(N_HID, N_HID)] * (N_LAYERS - 1) + [(N_OUT, N_HID)]
        pads = [(N_HID, PAD_IN)] + [(N_HID, N_HID)] * (N_LAYERS - 1) + [(PAD_OUT, N_HID)]
        f32 = dict(dtype=torch.float32, device=self.dev)
        self.W, self.b, self.mW, self.vW, self.mb, self.vb = [], [], [], [], [], []
        self.W16, self.W16T = [], []
        for (o, i), (po, pi) in zip(dims, pads):
            w = torch.zeros(po, pi, dtype=torch.float32)
            w[:o, :i] = (torch.rand(o, i, generator=g) * 2 - 1) * math.sqrt(6.0 / (i + o))
            self.W.append(w.to(self.dev))
            self.b.append(torch.zeros(po, **f32))
            self.mW.append(torch.zeros(po, pi, **f32))
            self.vW.append(torch.zeros(po, pi, **f32))
            self.mb.append(torch.zeros(po, **f32))
            self.vb.append(torch.zeros(po, **f32))
            self.W16.append(self.W[-1].to(torch.bfloat16).contiguous())
            self.W16T.append(self.W[-1].t().contiguous().to(torch.bfloat16))
        self.dims, self.pads = dims, pads
        self.step_count = 0
        self._alloc(max_batch)

    def _alloc(self, B):
        torch = self.torch
        B = (B + 127) // 128 * 128
        self.max_batch = B
        bf = dict(dtype=torch.bfloat16, device=self.dev)
        f32 = dict(dtype=torch.float32, device=self.dev)
        self.X32 = torch.zeros(B, PAD_IN, **f32)
        self.Z = [torch.zeros(B, N_HID, **bf) for _ in range(N_LAYERS)]
        self.H = [torch.zeros(B, N_HID, **bf) for _ in range(N_LAYERS)]
        self.HT = [torch.zeros(N_HID, B, **bf) for _ in range(N_LAYERS)]
        self.Y = torch.zeros(B, PAD_OUT, **f32)
        self.dZ = [torch.zeros(B, N_HID, **bf) for _ in range(N_LAYERS)]
        self.dZT = [torch.zeros(N_HID, B, **bf) for _ in range(N_LAYERS)]
        self.dY16 = torch.zeros(B, PAD_OUT, **bf)
        self.dYT16 = torch.zeros(PAD_OUT, B, **bf)
        self.sq = torch.zeros(B, **f32)
        self.T = torch.zeros(B, N_OUT, **f32)
        self.splits = 64
        self.part = torch.zeros(self.splits * N_HID * N_HID, **f32)
        self.gW = [torch.zeros_like(w) for w in self.W]
        self.gb = [torch.zeros_like(b) for b in self.b]

    # -- forward / backward -------------------------------------------------------------------------
    def _load_inputs(self, X):
        torch = self.torch
        n = X.shape[0]
        Bp = (n + 127) // 128 * 128
        if Bp > self.max_batch:
            self._alloc(Bp)
        x = torch.as_tensor(X, dtype=torch.float32, device=self.dev)
        self.X32[:n, :N_IN] = x
        if Bp > n:
            self.X32[n:Bp].zero_()
        return n, Bp

    def forward(self, X):
        """Network outputs (scaled space) for inputs X [n, 5]; returns a float32 tensor [n, 10]."""
        n, Bp = self._load_inputs(X)
        self._forward(Bp)
        return self.Y[:n, :N_OUT]

    def forward_fused(self, n):
        """Inference on the first n rows of self.X32 by the fused kernel (xd_mlp_forward): one
        persistent launch for the whole network; outputs (scaled space) in self.Y[:n]."""
        k = self.k
        net = _native.XdMlpNet()
        net.n_in, net.w1, net.ldw1 = N_IN, self.W[0].data_ptr(), PAD_IN
        for l in range(3):
            net.w[l] = self.W16[l + 1].data_ptr()
        net.w5 = self.W16[N_LAYERS].data_ptr()
        for l in range(5):
            net.b[l] = self.b[l].data_ptr()
        _native.check(k.lib.xd_mlp_forward(ctypes.byref(net), int(n), _p(self.X32), PAD_IN, _p(self.Y), PAD_OUT,
                                           _p(k.err), 0, k.stream()), "xd_mlp_forward")
        return self.Y[:n, :N_OUT]

    def _forward(self, Bp):
        k = self.k
        _native.check(k.lib.xd_mlp_input_layer(Bp, N_IN, N_HID, _p(self.X32), PAD_IN, _p(self.W[0]), PAD_IN,
                                               _p(self.b[0]), _p(self.Z[0]), _p(self.H[0]), _p(self.HT[0]),
                                               self.max_batch, k.stream()), "xd_mlp_input_layer")
        A, lda = self.H[0], N_HID
        for l in range(1, N_LAYERS):
            k.gemm(A, self.W16[l], Bp, N_HID, lda, lda, lda, EPI_BIAS_SILU, 128, bias=self.b[l], Z=self.Z[l],
                   H=self.H[l], HT=self.HT[l], ldc=N_HID, ldt=self.max_batch)
            A, lda = self.H[l], N_HID
        k.gemm(A, self.W16[N_LAYERS], Bp, PAD_OUT, N_HID, N_HID, N_HID, EPI_BIAS_F32, 16, C32=self.Y,
               bias=self.b[N_LAYERS], ldc=PAD_OUT)

    def _weight_grad(self, dZT, inT, n_out_rows, n_in, Bp, out):
        """out [n_out_rows x n_in] = dZT [rows x Bp] . inT [n_in x Bp]^T, split over the batch."""
        k = self.k
        tile_n = 16 if n_in <= 16 else 128
        splits = max(1, min(self.splits, Bp // 128))
        used = k.gemm(dZT, inT, n_out_rows, n_in, Bp, self.max_batch, self.max_batch, EPI_F32, tile_n, C32=self.part,
                      ldc=n_in, splits=splits)
        _native.check(k.lib.xd_splitk_sum(n_out_rows * n_in, used, _p(self.part), _p(out), k.stream()),
                      "xd_splitk_sum")

    def backward(self, n, Bp):
        """Gradients of the mean squared error (scaled space) w.r.t. every parameter, after a
        forward pass on a batch whose targets are in self.T[:n]."""
        k = self.k
        L = N_LAYERS
        scale = 2.0 / (n * N_OUT)
        _native.check(k.lib.xd_mse_grad(n, N_OUT, PAD_OUT, _p(self.Y), _p(self.T), ctypes.c_float(scale),
                                        _p(self.dY16), _p(self.dYT16), self.max_batch, _p(self.sq), k.stream()),
                      "xd_mse_grad")
        if Bp > n:
            self.dY16[n:Bp].zero_()
            self.dYT16[:, n:Bp].zero_()
        # Output layer.
        self._weight_grad(self.dYT16, self.HT[L - 1], PAD_OUT, N_HID, Bp, self.gW[L])
        _native.check(k.lib.xd_bias_grad(Bp, PAD_OUT, _p(self.dYT16), self.max_batch, _p(self.gb[L]), k.stream()),
                      "xd_bias_grad")
        k.gemm(self.dY16, self.W16T[L], Bp, N_HID, PAD_OUT, PAD_OUT, PAD_OUT, EPI_SILU_BACK, 128, Zin=self.Z[L - 1],
               H=self.dZ[L - 1], HT=self.dZT[L - 1], ldc=N_HID, ldt=self.max_batch)
        # Hidden layers L-1 .. 1 (weights W[l], l >= 1).
        for l in range(L - 1, 0, -1):
            self._weight_grad(self.dZT[l], self.HT[l - 1], N_HID, N_HID, Bp, self.gW[l])
            _native.check(k.lib.xd_bias_grad(Bp, N_HID, _p(self.dZT[l]), self.max_batch, _p(self.gb[l]), k.stream()),
                          "xd_bias_grad")
            k.gemm(self.dZ[l], self.W16T[l], Bp, N_HID, N_HID, N_HID, N_HID, EPI_SILU_BACK, 128, Zin=self.Z[l - 1],
                   H=self.dZ[l - 1], HT=self.dZT[l - 1], ldc=N_HID, ldt=self.max_batch)
        # First layer (FP32 on the CUDA cores).
        _native.check(k.lib.xd_mlp_input_grad(Bp, N_IN, N_HID, _p(self.dZT[0]), self.max_batch, _p(self.X32), PAD_IN,
                                              _p(self.gW[0]), PAD_IN, k.stream()), "xd_mlp_input_grad")
        _native.check(k.lib.xd_bias_grad(Bp, N_HID, _p(self.dZT[0]), self.max_batch, _p(self.gb[0]), k.stream()),
                      "xd_bias_grad")

    def adam_step(self, cfg: AdamConfig):
        k = self.k
        self.step_count += 1
        t = self.step_count
        a = _native.XdAdamArgs(cfg.lr, cfg.beta1, cfg.beta2, cfg.eps, 1 - cfg.beta1 ** t, 1 - cfg.beta2 ** t)
        for l in range(N_LAYERS + 1):
            ro, ri = self.pads[l]
            _native.check(k.lib.xd_adam(ro, ri, _p(self.W[l]), _p(self.gW[l]), _p(self.mW[l]), _p(self.vW[l]),
                                        ctypes.byref(a), _p(self.W16[l]), _p(self.W16T[l]), ri, ro, k.stream()),
                          "xd_adam")
            _native.check(k.lib.xd_adam(1, ro, _p(self.b[l]), _p(self.gb[l]), _p(self.mb[l]), _p(self.vb[l]),
                                        ctypes.byref(a), None, None, 0, 0, k.stream()), "xd_adam")
        # Keep the padding of the first and last layers exactly zero.
        self.W[0][:, N_IN:].zero_()
        self.W16[0][:, N_IN:].zero_()
        self.W16T[0][N_IN:, :].zero_()
        self.W[N_LAYERS][N_OUT:, :].zero_()
        self.W16[N_LAYERS][N_OUT:, :].zero_()
        self.W16T[N_LAYERS][:, N_OUT:].zero_()
        self.b[N_LAYERS][N_OUT:].zero_()

    def train_step(self, X, T, cfg: AdamConfig):
        """One Adam step on a batch (X [n, 5], T [n, 10] in scaled space); returns the loss tensor."""
        torch = self.torch
        n, Bp = self._load_inputs(X)
        self.T[:n] = torch.as_tensor(T, dtype=torch.float32, device=self.dev)
        self._forward(Bp)
        self.backward(n, Bp)
        self.adam_step(cfg)
        return self.sq[:n].mean() / N_OUT

    def parameters_numpy(self):
        """(W, b) per layer as float64 arrays, unpadded: the FP32 first layer, the BF16 weights the
        tensor-core layers use, and the FP32 biases."""
        out = []
        for l, (o, i) in enumerate(self.dims):
            w = self.W[0] if l == 0 else self.W16[l].float()
            out.append((w[:o, :i].double().cpu().numpy(), self.b[l][:o].double().cpu().numpy()))
        return out


# ---- training data from the FP64 BSIM4 kernel, and the two-network surrogate ---------------------

# Staged-slot indices (xd_copy_stamps layout) of the ten targets, per instance with the source
# grounded: F at D; Q at G, D, B; dF_D/dV_G, dF_D/dV_D, dF_D/dV_B; dQ_G/dV_G, dQ_G/dV_D, dQ_G/dV_B.
_TARGET_SLOTS = (0, 4 + 1, 4 + 0, 4 + 3, 16 + 1, 16 + 0, 16 + 3, 32 + 5, 32 + 4, 32 + 7)


def bsim4_samples(n, pmos, seed=0, card=None, n_geom=1024, device=0, chunk=1 << 20):
    """n samples of the FP64 BSIM4 load (this package's kernel) at biases uniform in |V| <= 1.2 V
    and geometries uniform in L 30-500 nm, W 0.1-10 um (n_geom distinct (L, W) pairs, each
    instance drawing one). Returns (features [n, 5] float32, targets [n, 10] float64)."""
    import torch

    from .device import Bsim4Device, ModelCard, SolverFlags

    rng = np.random.default_rng(seed)
    gl = rng.uniform(30e-9, 500e-9, n_geom)
    gw = rng.uniform(0.1e-6, 10e-6, n_geom)
    Xs, Ys = [], []
    done = 0
    dev = None
    while done < n:
        m = min(chunk, n - done)
        if dev is None or dev.n != m:
            if dev is not None:
                dev.close()
            geo = rng.integers(0, n_geom, m)
            nodes = np.stack([3 * np.arange(m), 3 * np.arange(m) + 1, -np.ones(m, np.int64), 3 * np.arange(m) + 2], 1)
            rowptr = np.arange(0, 9 * m + 1, 3, dtype=np.int32)
            colind = (np.repeat(3 * np.arange(m), 9) + np.tile([0, 1, 2], 3 * m)).astype(np.int32)
            dev = Bsim4Device([card or ModelCard(pmos, {})], np.zeros(m, np.int32), nodes,
                              {"L": gl[geo], "W": gw[geo]}, (rowptr, colind), 3 * m, device=device)
            geo_l, geo_w = gl[geo], gw[geo]
        v = rng.uniform(-VMAX, VMAX, (m, 3))  # Vds, Vgs, Vbs with the source at ground
        sol = torch.as_tensor(v.reshape(-1), dtype=torch.float64, device=f"cuda:{device}")
        z = lambda k: torch.zeros(k, dtype=torch.float64, device=f"cuda:{device}")
        nsta, nsto = z(dev.n_state), z(dev.n_store)
        f, q, fx, qx = z(3 * m), z(3 * m), z(3 * m), z(3 * m)
        jf, jq = z(dev.nnz), z(dev.nnz)
        dev.load(SolverFlags(newton_iter=1, voltlim=0), sol, nsta, z(dev.n_state), nsto, z(dev.n_store), f, q, fx, qx,
                 jf, jq)
        st = dev.copy_stamps()
        Ys.append(st[list(_TARGET_SLOTS)].T.copy())
        Xs.append(features(v[:, 1], v[:, 0], v[:, 2], geo_w, geo_l).astype(np.float32))
        done += m
    if dev is not None:
        dev.close()
    return np.concatenate(Xs), np.concatenate(Ys)


def error_report(pred, ref):
    """Per output, over the samples whose reference magnitude is at least 1% of the output's RMS:
    median and 95th percentile of the relative error |pred - ref| / |ref|, and the fraction of all
    samples in that set."""
    out = {}
    for k, name in enumerate(OUTPUT_NAMES):
        rms = np.sqrt(np.mean(ref[:, k] ** 2)) or 1.0
        sel = np.abs(ref[:, k]) >= 0.01 * rms
        e = np.abs(pred[sel, k] - ref[sel, k]) / np.abs(ref[sel, k])
        out[name] = {"rel_median": float(np.median(e)), "rel_p95": float(np.quantile(e, 0.95)),
                     "fraction": float(sel.mean())}
    return out


class BsimSurrogate:
    """The NMOS and PMOS networks of the BSIM4 surrogate, trained on FP64 kernel samples."""

    def __init__(self, device=0, seed=0):
        self.device = device
        self.nets = {False: SurrogateMLP(device, seed=seed), True: SurrogateMLP(device, seed=seed + 1)}
        self.history = {False: [], True: []}

    def train(self, n_samples=10_000_000, epochs=8, batch=16384, lr=3e-3, lr_end=5e-5, seed=0, log=None):
        """Trains each type on n_samples FP64 samples; returns the held-out error report per type."""
        import torch

        reports = {}
        for pmos in (False, True):
            X, Y = bsim4_samples(n_samples + 200_000, pmos, seed=seed + (7 if pmos else 0), device=self.device)
            Xv, Yv = X[-200_000:], Y[-200_000:]
            X, Y = X[:-200_000], Y[:-200_000]
            T = encode_targets(Y).astype(np.float32)
            net = self.nets[pmos]
            Xd = torch.as_tensor(X, device=net.dev)
            Td = torch.as_tensor(T, device=net.dev)
            steps = epochs * (len(X) // batch)
            g = torch.Generator(device=net.dev).manual_seed(seed)
            s = 0
            for ep in range(epochs):
                perm = torch.randperm(len(X), device=net.dev, generator=g)
                for i in range(len(X) // batch):
                    idx = perm[i * batch:(i + 1) * batch]
                    cur = lr_end + 0.5 * (lr - lr_end) * (1 + math.cos(math.pi * s / max(1, steps)))
                    loss = net.train_step(Xd[idx], Td[idx], AdamConfig(lr=cur))
                    s += 1
                    if i % 200 == 0:
                        self.history[pmos].append((s, float(loss)))
                        if log:
                            log(f"{'pmos' if pmos else 'nmos'} epoch {ep} step {s}/{steps} loss {float(loss):.4g}")
            net.k.check_err()
            pred = self.predict_physical(pmos, Xv)
            reports["pmos" if pmos else "nmos"] = error_report(pred, Yv)
        return reports

    def predict_physical(self, pmos, X, batch=262144):
        out = []
        net = self.nets[pmos]
        for i in range(0, len(X), batch):
            n, _ = net._load_inputs(X[i:i + batch])
            out.append(net.forward_fused(n).double().cpu().numpy())
        return decode_outputs(np.concatenate(out))


class SurrogateLoads:
    """Vector loads (F, Q) of a circuit's BSIM4 family from the trained surrogate, on the GPU:
    inputs built from the solution by ``xd_surrogate_features``, both networks' forward passes,
    outputs decoded and staged by ``xd_surrogate_stage`` and assembled through the family's own
    gather map by ``xd_load_vectors_staged`` (stored, not added)."""

    def __init__(self, sur: BsimSurrogate, family, mos_type, mos_nodes, w, l):
        import torch

        self.torch = torch
        self.sur = sur
        self.fam = family
        self.dev = sur.nets[False].dev
        self.lib = _native.load()
        n = len(mos_type)
        self.n = n
        T = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=self.dev)
        self.nodes4 = T(np.asarray(mos_nodes, np.int32).reshape(-1), torch.int32)
        f = features(np.zeros(n), np.zeros(n), np.zeros(n), np.asarray(w, float), np.asarray(l, float))
        self.geom2 = T(f[:, 3:5].astype(np.float32).reshape(-1), torch.float32)
        self.idx = {p: T(np.nonzero(np.asarray(mos_type) == (1 if p else 0))[0].astype(np.int32), torch.int32)
                    for p in (False, True)}
        self.out_scale = T(OUTPUT_SCALE.astype(np.float32), torch.float32)
        self.stage = torch.zeros(16 * n, dtype=torch.float64, device=self.dev)
        for p in (False, True):
            m = int(self.idx[p].shape[0])
            net = sur.nets[p]
            if m > net.max_batch:
                net._alloc(m)

    def load(self, x, f, q, fx, qx, stream):
        for p in (False, True):
            m = int(self.idx[p].shape[0])
            if m == 0:
                continue
            net = self.sur.nets[p]
            _native.check(self.lib.xd_surrogate_features(m, _p(self.idx[p]), _p(self.nodes4), _p(x), _p(self.geom2),
                                                         ctypes.c_float(VMAX), _p(net.X32), PAD_IN, stream),
                          "xd_surrogate_features")
            net.forward_fused(m)
            _native.check(self.lib.xd_surrogate_stage(m, _p(self.idx[p]), _p(net.Y), PAD_OUT, _p(self.out_scale),
                                                      self.n, _p(self.stage), stream), "xd_surrogate_stage")
        _native.check(self.lib.xd_load_vectors_staged(self.fam._h, _p(self.stage), _p(f), _p(q), _p(fx), _p(qx), 1,
                                                      stream), "xd_load_vectors_staged")
