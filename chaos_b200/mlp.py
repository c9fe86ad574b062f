"""The learned screen's network: a BF16 MLP (FP32 accumulation) trained and run by this library's own tensor-core
kernels (`cl_b200_gemm_bf16`: tcgen05.mma with a tensor-memory accumulator) and elementwise kernels (cl_mlp.cu).

64 inputs -> 256 -> 256 -> 256 (GELU, tanh form) -> 2 outputs: the logit of P(chaotic) and a prediction of the
final lambda_1. Inference runs the whole network in one persistent tensor-core kernel (`cl_b200_mlp_forward_fused`)
on weights packed once into the MMA layout; training runs it layer by layer, keeping the pre-activations. No reference counterpart: the reference has no learned component. PyTorch only holds the device buffers
and the stream; every arithmetic step runs in the library's kernels.

Training is mean binary cross-entropy on the label plus `w_reg` times the mean squared error on lambda_1, with Adam
on FP32 master weights whose BF16 copies (and their transposes, for the backward GEMMs) feed the tensor cores.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from ._lib import last_error, lib

DIMS = (64, 256, 256, 256, 2)
OUT_PAD = 16   # the last layer's 2 outputs padded to the smallest tensor-core N tile


def _ck(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what}: {rc} {last_error()}")


def _declare(L):
    if getattr(L, "_mlp_declared", False):
        return L
    vp, f32p = C.c_void_p, C.c_void_p
    L.cl_b200_gemm_bf16.argtypes = [vp, C.c_int32, vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, f32p, C.c_int32,
                                    f32p, vp, C.c_int32, f32p, C.c_int32, vp]
    L.cl_b200_transpose_bf16.argtypes = [vp, C.c_int32, C.c_int32, C.c_int32, vp, C.c_int32, vp]
    L.cl_b200_gelu_backward.argtypes = [f32p, f32p, C.c_int64, vp, f32p, vp]
    L.cl_b200_col_sum.argtypes = [f32p, C.c_int32, C.c_int32, C.c_int32, f32p, vp]
    L.cl_b200_head_loss.argtypes = [f32p, C.c_int32, C.c_int32, f32p, f32p, C.c_float, f32p, vp, f32p, vp]
    L.cl_b200_adam.argtypes = [f32p, f32p, f32p, f32p, C.c_int64, C.c_float, C.c_float, C.c_float, C.c_float,
                               C.c_int32, vp, vp, C.c_int32, C.c_int32, vp]
    L.cl_b200_to_bf16.argtypes = [f32p, C.c_int64, vp, vp]
    L.cl_b200_screen_features.argtypes = [vp, C.c_int64, C.c_int64, C.c_int32, C.c_int32, f32p, vp, vp]
    L.cl_b200_mlp_status.argtypes = []
    L.cl_b200_mlp_pack_kmajor.argtypes = [vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, vp, vp]
    L.cl_b200_mlp_forward_fused.argtypes = [vp, C.c_int32, vp, vp, vp, vp, f32p, f32p, f32p, f32p, f32p, C.c_int32, vp]
    for nm in ("cl_b200_mlp_pack_kmajor", "cl_b200_mlp_forward_fused", "cl_b200_gemm_bf16", "cl_b200_transpose_bf16", "cl_b200_gelu_backward", "cl_b200_col_sum",
               "cl_b200_head_loss", "cl_b200_adam", "cl_b200_to_bf16", "cl_b200_screen_features",
               "cl_b200_mlp_status"):
        getattr(L, nm).restype = C.c_int
    L._mlp_declared = True
    return L


def gemm(A, B, M, N, K, *, bias=None, gelu=False, C32=None, Cb=None, pre=None, accumulate=False, stream=None):
    """C = A . B^T (+ bias) (GELU) on the tensor cores; A (M x K) and B (N x K) row-major BF16 torch tensors."""
    L = _declare(lib())
    ldc = (C32 if C32 is not None else Cb).shape[1]
    p = lambda t: None if t is None else t.data_ptr()  # noqa: E731
    _ck(L.cl_b200_gemm_bf16(A.data_ptr(), A.shape[1], B.data_ptr(), B.shape[1], M, N, K, p(bias), int(gelu), p(C32),
                            p(Cb), ldc, p(pre), int(accumulate), stream), "gemm")


class MLP:
    """Weights (FP32 masters + BF16 copies and transposes) and the forward / backward passes on the device."""

    def __init__(self, torch, device, seed: int = 0, dims=DIMS):
        self.t, self.dev, self.dims = torch, device, dims
        g = np.random.default_rng(seed)
        self.layers = []
        for li in range(len(dims) - 1):
            fin, fout = dims[li], dims[li + 1]
            rows = OUT_PAD if li == len(dims) - 2 else fout
            W = np.zeros((rows, fin), np.float32)
            W[:fout] = g.normal(0.0, math.sqrt(2.0 / fin), (fout, fin)).astype(np.float32)
            if li == len(dims) - 2:
                W[:fout] *= 0.1
            b = np.zeros(rows, np.float32)
            self.layers.append(self._layer(W, b))
        self.step = 0

    def _layer(self, W, b):
        t, d = self.t, self.dev
        Wt = t.tensor(W, device=d)
        lay = dict(W=Wt, b=t.tensor(b, device=d), Wb=t.empty(W.shape, dtype=t.bfloat16, device=d),
                   Wbt=t.empty((W.shape[1], W.shape[0]), dtype=t.bfloat16, device=d),
                   mW=t.zeros_like(Wt), vW=t.zeros_like(Wt), mb=t.zeros(len(b), device=d), vb=t.zeros(len(b), device=d),
                   gW=t.zeros_like(Wt), gb=t.zeros(len(b), device=d))
        self._refresh(lay)
        return lay

    def _refresh(self, lay):
        L = _declare(lib())
        n = lay["W"].numel()
        _ck(L.cl_b200_to_bf16(lay["W"].data_ptr(), n, lay["Wb"].data_ptr(), self.stream()), "to bf16")
        r, c = lay["W"].shape
        _ck(L.cl_b200_transpose_bf16(lay["Wb"].data_ptr(), r, c, c, lay["Wbt"].data_ptr(), r, self.stream()), "transpose")

    def stream(self):
        return self.t.cuda.current_stream(self.dev).cuda_stream

    def packed(self):
        """The BF16 weights packed into the tensor cores' K-major tiles (rows = each layer's output rows), made once
        per weight update."""
        if getattr(self, "_packed", None) is not None and self._packed[0] == self.step:
            return self._packed[1]
        L, t = _declare(lib()), self.t
        out = []
        for lay in self.layers:
            r, c = lay["Wb"].shape
            buf = t.empty(r * ((c + 63) // 64) * 64, dtype=t.bfloat16, device=self.dev)
            _ck(L.cl_b200_mlp_pack_kmajor(lay["Wb"].data_ptr(), r, c, c, r, buf.data_ptr(), self.stream()), "pack")
            out.append(buf)
        self._packed = (self.step, out)
        return out

    def forward_fused(self, Xb, out=None, max_ctas: int = 0):
        """Inference: Xb (B, 64) BF16 contiguous -> FP32 outputs (B, 16) in one kernel, bit for bit `forward`."""
        if self.dims != DIMS:
            raise ValueError("the fused pass is built for the screen network's shape 64-256-256-256-16")
        t, L = self.t, _declare(lib())
        Xb = Xb.contiguous()
        B = Xb.shape[0]
        if out is None:
            out = t.empty((B, OUT_PAD), dtype=t.float32, device=self.dev)
        P = self.packed()
        b = [lay["b"] for lay in self.layers]
        _ck(L.cl_b200_mlp_forward_fused(Xb.data_ptr(), B, *[p.data_ptr() for p in P], *[x.data_ptr() for x in b],
                                        out.data_ptr(), int(max_ctas), self.stream()), "fused forward")
        return out

    def forward_fused_host(self, Xh, out_h, chunk_rows: int = 65536):
        """Inference from and to host memory: Xh (B, 64) BF16 and out_h (B, 16) FP32, pinned CPU tensors. The rows go
        in chunks over two streams, so the copies of one chunk (host to device, then the outputs back) overlap the
        fused pass over the other; the outputs are those of `forward_fused`, bit for bit. Returns out_h once the
        current stream has them (synchronise it before reading)."""
        if self.dims != DIMS:
            raise ValueError("the fused pass is built for the screen network's shape 64-256-256-256-16")
        t, L = self.t, _declare(lib())
        B = Xh.shape[0]
        P = self.packed()
        pp = [p.data_ptr() for p in P] + [lay["b"].data_ptr() for lay in self.layers]
        cur = t.cuda.current_stream(self.dev)
        streams = [t.cuda.Stream(self.dev) for _ in range(2)]
        rows = min(chunk_rows, max(B, 1))
        bufs = [(t.empty((rows, 64), dtype=t.bfloat16, device=self.dev),
                 t.empty((rows, OUT_PAD), dtype=t.float32, device=self.dev)) for _ in streams]
        for s_, (xd, od) in zip(streams, bufs):
            s_.wait_stream(cur)             # the weights and inputs the caller enqueued before
            xd.record_stream(s_)
            od.record_stream(s_)
        for i, lo in enumerate(range(0, B, rows)):
            s_ = streams[i % 2]
            xd, od = bufs[i % 2]
            n = min(B, lo + rows) - lo
            with t.cuda.stream(s_):
                xd[:n].copy_(Xh[lo:lo + n], non_blocking=True)
                _ck(L.cl_b200_mlp_forward_fused(xd.data_ptr(), n, *pp, od.data_ptr(), 0, s_.cuda_stream),
                    "fused forward")
                out_h[lo:lo + n].copy_(od[:n], non_blocking=True)
        for s_ in streams:
            cur.wait_stream(s_)
        return out_h

    def weights_numpy(self):
        return [(l["W"].cpu().numpy().copy(), l["b"].cpu().numpy().copy()) for l in self.layers]

    def forward(self, Xb, keep: bool = False):
        """Xb: (B, 64) BF16, B a multiple of 128. Returns the FP32 outputs (B, 16); with keep, the activations."""
        t = self.t
        B = Xb.shape[0]
        acts, pres = [Xb], []
        A = Xb
        nl = len(self.layers)
        for li, lay in enumerate(self.layers):
            rows, fin = lay["W"].shape
            last = li == nl - 1
            pre = t.empty((B, rows), dtype=t.float32, device=self.dev) if (keep and not last) else None
            if last:
                out = t.empty((B, rows), dtype=t.float32, device=self.dev)
                gemm(A, lay["Wb"], B, rows, fin, bias=lay["b"], C32=out, stream=self.stream())
                acts.append(out)
            else:
                Ab = t.empty((B, rows), dtype=t.bfloat16, device=self.dev)
                gemm(A, lay["Wb"], B, rows, fin, bias=lay["b"], gelu=True, Cb=Ab, pre=pre, stream=self.stream())
                acts.append(Ab)
                A = Ab
            pres.append(pre)
        if keep:
            self._acts, self._pres = acts, pres
        return acts[-1]

    def backward(self, dout32, doutb):
        """dout: dL/d(outputs) (B, 16) in FP32 and BF16; fills each layer's gW, gb."""
        t, L = self.t, _declare(lib())
        B = dout32.shape[0]
        dZ32, dZb = dout32, doutb
        for li in range(len(self.layers) - 1, -1, -1):
            lay = self.layers[li]
            rows, fin = lay["W"].shape
            Aprev = self._acts[li]                                 # (B, fin) BF16
            # dW = dZ^T . A_prev: M = rows, N = fin, K = B (both operands transposed to K-major)
            dZt = t.empty((rows, B), dtype=t.bfloat16, device=self.dev)
            _ck(L.cl_b200_transpose_bf16(dZb.data_ptr(), B, rows, dZb.shape[1], dZt.data_ptr(), B, self.stream()), "T")
            At = t.empty((fin, B), dtype=t.bfloat16, device=self.dev)
            _ck(L.cl_b200_transpose_bf16(Aprev.data_ptr(), B, fin, Aprev.shape[1], At.data_ptr(), B, self.stream()), "T")
            gemm(dZt, At, rows, fin, B, C32=lay["gW"], stream=self.stream())
            _ck(L.cl_b200_col_sum(dZ32.data_ptr(), B, rows, dZ32.shape[1], lay["gb"].data_ptr(), self.stream()), "db")
            if li == 0:
                break
            # dA_prev = dZ . W: M = B, N = fin, K = rows (W^T copy is the K-major operand)
            dA = t.empty((B, fin), dtype=t.float32, device=self.dev)
            gemm(dZb, lay["Wbt"], B, fin, rows, C32=dA, stream=self.stream())
            pre = self._pres[li - 1]
            dZ32 = t.empty((B, fin), dtype=t.float32, device=self.dev)
            dZb = t.empty((B, fin), dtype=t.bfloat16, device=self.dev)
            _ck(L.cl_b200_gelu_backward(dA.data_ptr(), pre.data_ptr(), dA.numel(), dZb.data_ptr(), dZ32.data_ptr(),
                                        self.stream()), "gelu backward")

    def loss_and_grad(self, out, label, target, w_reg):
        t, L = self.t, _declare(lib())
        B, ld = out.shape
        g32 = t.empty_like(out)
        gb = t.empty(out.shape, dtype=t.bfloat16, device=self.dev)
        rl = t.empty(B, dtype=t.float32, device=self.dev)
        _ck(L.cl_b200_head_loss(out.data_ptr(), B, ld, label.data_ptr(), target.data_ptr(), w_reg, g32.data_ptr(),
                                gb.data_ptr(), rl.data_ptr(), self.stream()), "head loss")
        return rl, g32, gb

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        L = _declare(lib())
        self.step += 1
        for lay in self.layers:
            r, c = lay["W"].shape
            _ck(L.cl_b200_adam(lay["W"].data_ptr(), lay["gW"].data_ptr(), lay["mW"].data_ptr(), lay["vW"].data_ptr(),
                               lay["W"].numel(), lr, b1, b2, eps, self.step, lay["Wb"].data_ptr(), lay["Wbt"].data_ptr(),
                               r, c, self.stream()), "adam W")
            _ck(L.cl_b200_adam(lay["b"].data_ptr(), lay["gb"].data_ptr(), lay["mb"].data_ptr(), lay["vb"].data_ptr(),
                               lay["b"].numel(), lr, b1, b2, eps, self.step, None, None, 1, lay["b"].numel(),
                               self.stream()), "adam b")

    def train_step(self, Xb, label, target, w_reg=1.0, lr=1e-3):
        out = self.forward(Xb, keep=True)
        rl, g32, gb = self.loss_and_grad(out, label, target, w_reg)
        self.backward(g32, gb)
        self.adam(lr=lr)
        return rl

    def predict(self, Xb):
        """Outputs (n, 16) FP32 for every row of Xb: column 0 the chaos logit (P = sigmoid), column 1 the lambda_1
        prediction. One fused launch over all rows."""
        return self.forward_fused(Xb)
