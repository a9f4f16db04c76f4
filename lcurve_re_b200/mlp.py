"""The surrogate network: nin -> 4 x 256 GELU -> nout, trained and evaluated on
this library's kernels (lcg_mlp_*), with torch tensors as device storage.

Layer 0 (nin <= 16 inputs) runs in FP32 on the CUDA cores, so the physical
parameters enter unrounded; layers 1-3 (256 -> 256, GELU) and the output
layer (256 -> nout, linear) are BF16 tensor-core GEMMs with FP32
accumulation and fused epilogues. Weights are FP32 masters updated by Adam,
with BF16 copies and BF16 transposes written by the optimiser step for the
forward and backward GEMMs. The loss is the mean squared error over the
outputs.

Batches are padded to a multiple of 128 rows; training steps use full
batches.
"""
import ctypes as C

import numpy as np

from . import abi
from .engine import load_library

EPI_GELU, EPI_LINEAR, EPI_DGELU, EPI_F32 = 0, 1, 2, 3


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


class MLP:
    def __init__(self, nin=9, nout=64, width=256, depth=4, batch=4096, device="cuda", seed=0):
        import torch
        if nin > 16 or width % 256 or nout % 64 or nout > 256:
            raise ValueError("nin <= 16, width a multiple of 256, nout a multiple of 64 <= 256")
        self.torch = torch
        self.lib = load_library()
        self.nin, self.nout, self.width, self.depth = nin, nout, width, depth
        self.B = ((batch + 127) // 128) * 128
        self.dev = torch.device(device)
        g = torch.Generator(device="cpu").manual_seed(seed)
        f32 = dict(dtype=torch.float32, device=self.dev)
        b16 = dict(dtype=torch.bfloat16, device=self.dev)
        # layers: 0 input (FP32), 1..depth-1 hidden, depth output
        shapes = [(width, nin)] + [(width, width)] * (depth - 1) + [(nout, width)]
        self.W, self.b = [], []
        for (o, i) in shapes:
            w = torch.randn(o, i, generator=g) * np.sqrt(2.0 / i)
            self.W.append(w.to(**f32).contiguous())
            self.b.append(torch.zeros(o, **f32))
        self.Wb = [None] + [w.to(torch.bfloat16).contiguous() for w in self.W[1:]]
        self.Wt = [None] + [w.t().contiguous().to(torch.bfloat16) for w in self.W[1:]]
        self.mW = [torch.zeros_like(w) for w in self.W]
        self.vW = [torch.zeros_like(w) for w in self.W]
        self.mb = [torch.zeros_like(b) for b in self.b]
        self.vb = [torch.zeros_like(b) for b in self.b]
        self.dW = [torch.zeros(o if o >= 128 else 128, i, **f32) for (o, i) in shapes]
        self.db = [torch.zeros(o, **f32) for (o, _) in shapes]
        B = self.B
        self.x = torch.zeros(B, nin, **f32)
        self.Z = [torch.zeros(B, width, **b16) for _ in range(depth)]
        self.Y = [torch.zeros(B, width, **b16) for _ in range(depth)]
        self.Yt = [torch.zeros(width, B, **b16) for _ in range(depth)]
        self.out = torch.zeros(B, nout, **f32)
        self.G = [torch.zeros(B, width, **b16) for _ in range(depth)] + \
                 [torch.zeros(B, nout, **b16)]
        self.Gt = [torch.zeros(width, B, **b16) for _ in range(depth)] + \
                  [torch.zeros(max(nout, 128), B, **b16)]
        self.loss_rows = torch.zeros(B, **f32)
        self.err = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self.step_no = 0

    # -- plumbing --------------------------------------------------------------
    def _stream(self):
        return C.c_void_p(self.torch.cuda.current_stream(self.dev).cuda_stream)

    def _ok(self, st, what):
        if st != abi.OK:
            raise RuntimeError("%s failed with status %d" % (what, st))

    def _gemm(self, epi, m, n, k, a, b, bias=None, z=None, y=None, yt=None, out=None,
              mvalid=None, ldt=None):
        self._ok(self.lib.lcg_mlp_gemm(self._stream(), epi, m, n, k, _p(a), _p(b), _p(bias),
                                       _p(z), _p(y), _p(yt), _p(out),
                                       m if mvalid is None else mvalid,
                                       0 if ldt is None else ldt, _p(self.err)), "lcg_mlp_gemm")

    # -- forward / backward ----------------------------------------------------
    def forward(self, x, train=False):
        """x: [n, nin] FP32 device tensor (n <= batch). Returns the [n, nout]
        FP32 outputs (a view of an internal buffer). Training runs the whole
        batch; inference only the first n rows rounded up to the 128-row
        tile of the GEMMs."""
        n = x.shape[0]
        if n > self.B:
            raise ValueError("batch larger than the network's buffers")
        B, w = self.B, self.width
        m = B if train else min(B, max(128, (n + 127) // 128 * 128))
        self.x[:n].copy_(x)
        if n < m:
            self.x[n:m].zero_()
        st = self.lib.lcg_mlp_input(self._stream(), _p(self.x), self.nin, _p(self.W[0]),
                                    _p(self.b[0]), m, w, n, _p(self.Z[0]), _p(self.Y[0]),
                                    _p(self.Yt[0]) if train else None, B)
        self._ok(st, "lcg_mlp_input")
        for l in range(1, self.depth):
            self._gemm(EPI_GELU, m, w, w, self.Y[l - 1], self.Wb[l], bias=self.b[l], z=self.Z[l],
                       y=self.Y[l], yt=self.Yt[l] if train else None, mvalid=m, ldt=B)
        L = self.depth
        self._gemm(EPI_LINEAR, m, self.nout, w, self.Y[L - 1], self.Wb[L], bias=self.b[L],
                   out=self.out, mvalid=n)
        return self.out[:n]

    def backward(self, target):
        """Gradients of the mean squared error of the last forward (a full
        training batch) against target [B, nout]; returns the loss."""
        B, w, L = self.B, self.width, self.depth
        st = self.lib.lcg_mlp_mse_grad(self._stream(), _p(self.out), _p(target), B, self.nout,
                                       B, B, _p(self.G[L]), _p(self.Gt[L]), _p(self.loss_rows))
        self._ok(st, "lcg_mlp_mse_grad")
        # output layer
        self._gemm(EPI_F32, self.Gt[L].shape[0], w, B, self.Gt[L], self.Yt[L - 1],
                   out=self.dW[L], mvalid=self.nout)
        self._colsum(self.G[L], self.nout, self.db[L])
        self._gemm(EPI_DGELU, B, w, self.nout, self.G[L], self.Wt[L], z=self.Z[L - 1],
                   y=self.G[L - 1], yt=self.Gt[L - 1], mvalid=B, ldt=B)
        for l in range(L - 1, 0, -1):
            self._gemm(EPI_F32, w, w, B, self.Gt[l], self.Yt[l - 1], out=self.dW[l], mvalid=w)
            self._colsum(self.G[l], w, self.db[l])
            self._gemm(EPI_DGELU, B, w, w, self.G[l], self.Wt[l], z=self.Z[l - 1],
                       y=self.G[l - 1], yt=self.Gt[l - 1] if l > 1 else None, mvalid=B, ldt=B)
        st = self.lib.lcg_mlp_input_grad(self._stream(), _p(self.G[0]), _p(self.x), self.nin, B,
                                         w, B, _p(self.dW[0]))
        self._ok(st, "lcg_mlp_input_grad")
        self._colsum(self.G[0], w, self.db[0])
        return float(self.loss_rows.sum().item()) / (B * self.nout)

    def _colsum(self, g, cols, out):
        self._ok(self.lib.lcg_mlp_colsum(self._stream(), _p(g), self.B, cols, self.B, _p(out)),
                 "lcg_mlp_colsum")

    def step(self, lr, beta1=0.9, beta2=0.999, eps=1e-8):
        """One Adam step on every weight and bias."""
        self.step_no += 1
        s = self._stream()
        for l in range(self.depth + 1):
            o, i = self.W[l].shape
            st = self.lib.lcg_mlp_adam(s, _p(self.W[l]), _p(self.mW[l]), _p(self.vW[l]),
                                       _p(self.dW[l]), o, i, lr, beta1, beta2, eps, self.step_no,
                                       _p(self.Wb[l]), _p(self.Wt[l]))
            self._ok(st, "lcg_mlp_adam")
            st = self.lib.lcg_mlp_adam(s, _p(self.b[l]), _p(self.mb[l]), _p(self.vb[l]),
                                       _p(self.db[l]), 1, o, lr, beta1, beta2, eps, self.step_no,
                                       None, None)
            self._ok(st, "lcg_mlp_adam")

    def check(self):
        """Raises if a kernel reported a pipeline timeout."""
        if int(self.err.item()) != 0:
            raise RuntimeError("tensor-core pipeline wait timed out (code %d)" % int(self.err.item()))

    def flops_per_sample(self, train=False):
        f = 2 * (self.nin * self.width + (self.depth - 1) * self.width ** 2 +
                 self.width * self.nout)
        return 3 * f if train else f

    # -- state -----------------------------------------------------------------
    def state(self):
        return {"W%d" % l: self.W[l].cpu().numpy() for l in range(self.depth + 1)} | \
               {"b%d" % l: self.b[l].cpu().numpy() for l in range(self.depth + 1)}

    def load_state(self, st):
        torch = self.torch
        for l in range(self.depth + 1):
            self.W[l].copy_(torch.as_tensor(st["W%d" % l]))
            self.b[l].copy_(torch.as_tensor(st["b%d" % l]))
            if l > 0:
                self.Wb[l].copy_(self.W[l].to(torch.bfloat16))
                self.Wt[l].copy_(self.W[l].t().to(torch.bfloat16))
