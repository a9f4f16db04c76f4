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


def _ptrs(ts):
    """A ctypes array of the tensors' device pointers (NULL for None)."""
    return (C.c_void_p * len(ts))(*[t.data_ptr() if t is not None else None for t in ts])


def _split_operand(x, rows, kp, order):
    """[rows x 3 kp] BF16: the three K-blocks of x = hi + lo in the given
    order ('h' or 'l' each), zero-padded to rows x kp per block."""
    import torch
    hi = x.to(torch.bfloat16)
    lo = (x - hi.to(x.dtype)).to(torch.bfloat16)
    out = torch.zeros(rows, 3 * kp, dtype=torch.bfloat16, device=x.device)
    n, k = x.shape
    for j, part in enumerate(order):
        out[:n, j * kp:j * kp + k] = hi if part == "h" else lo
    return out


def gemm_bf16x3(a, b, lib=None, kblock=8192):
    """a @ b.T (a [M x K], b [N x K], FP32 or FP64 device tensors) as an FP64
    [M x N] tensor whose products run on the tensor cores (lcg_mlp_gemm).

    Each operand is split as x = hi + lo with hi = bf16(x) and
    lo = bf16(x - hi), which represents x to about 2^-17 of its magnitude,
    and the three leading products hi_a hi_b + lo_a hi_b + hi_a lo_b run as
    one BF16 GEMM with FP32 accumulation over the concatenated K
    (A = [hi | lo | hi], B = [hi | hi | lo]); the dropped lo_a lo_b term is
    below 2^-18 of each product (the bfloat16x3 scheme of Henry, Tang and
    Heinecke, 2019). K is cut into blocks of kblock, one GEMM each, whose
    FP32 results are summed in FP64, so the FP32 accumulation error stays
    that of kblock terms however long K is. Sizes are padded with zeros to
    the kernel's tiles."""
    import torch
    lib = lib or load_library()
    if a.shape[1] != b.shape[1]:
        raise ValueError("a and b need the same K")
    M, K = a.shape
    N = b.shape[0]
    mp, np_ = -(-M // 128) * 128, -(-N // 64) * 64
    stream = C.c_void_p(torch.cuda.current_stream(a.device).cuda_stream)
    acc = torch.zeros(M, N, dtype=torch.float64, device=a.device)
    out = torch.empty(M, np_, dtype=torch.float32, device=a.device)
    for k0 in range(0, K, kblock):
        k1 = min(K, k0 + kblock)
        kp = -(-(k1 - k0) // 256) * 256
        A = _split_operand(a[:, k0:k1], mp, kp, "hlh")
        B = _split_operand(b[:, k0:k1], np_, kp, "hhl")
        st = lib.lcg_mlp_gemm(stream, EPI_F32, mp, np_, 3 * kp, _p(A), _p(B), None, None, None,
                              None, _p(out), M, 0, None)
        if st != abi.OK:
            raise RuntimeError("lcg_mlp_gemm failed with status %d" % st)
        acc += out[:, :N]
    return acc


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
        # the one-launch chains (lcg_mlp_forward / lcg_mlp_backward_data) hold
        # a 256-wide tile; other widths run layer by layer
        self.fused = width == 256 and depth <= 5
        L = depth
        self._fw_w = _ptrs(self.Wb[1:])
        self._fw_b = _ptrs(self.b[1:])
        self._fw_z = _ptrs(self.Z)
        self._fw_yt = _ptrs(self.Yt)
        self._bw_wt = _ptrs([self.Wt[l] for l in range(L, 0, -1)])
        self._bw_z = _ptrs([self.Z[l] for l in range(L - 1, -1, -1)])
        self._bw_g = _ptrs([self.G[l] for l in range(L - 1, -1, -1)])
        self._bw_gt = _ptrs([self.Gt[l] for l in range(L - 1, 0, -1)] + [None])
        self._target_fused = False
        # graph-captured training steps: static batch, device-side schedule
        self.tgt = torch.zeros(B, nout, **f32)
        self.sched = torch.tensor([1e-3, 1e-3, 0.0, 0.9, 0.999, 1e-8], **f32)
        self.step_dev = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self.loss_acc = torch.zeros(1, dtype=torch.float64, device=self.dev)
        ts = [(self.W[l], self.mW[l], self.vW[l], self.dW[l], self.Wb[l], self.Wt[l])
              for l in range(L + 1)] + \
             [(self.b[l], self.mb[l], self.vb[l], self.db[l], None, None) for l in range(L + 1)]
        self._adam = [len(ts)] + [_ptrs([t[i] for t in ts]) for i in range(6)]
        self._adam_rows = (C.c_int32 * len(ts))(*[t[0].shape[0] if t[0].dim() == 2 else 1
                                                  for t in ts])
        self._adam_cols = (C.c_int32 * len(ts))(*[t[0].shape[-1] for t in ts])
        self._graph = None

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
    def forward(self, x, train=False, target=None):
        """x: [n, nin] FP32 device tensor (n <= batch). Returns the [n, nout]
        FP32 outputs (a view of an internal buffer). Training runs the whole
        batch; inference only the first n rows rounded up to the 128-row
        tile. With target ([batch, nout] FP32, training only) the fused
        chain also forms the loss gradient, so backward() needs no target."""
        n = x.shape[0]
        if n > self.B:
            raise ValueError("batch larger than the network's buffers")
        B, w = self.B, self.width
        m = B if train else min(B, max(128, (n + 127) // 128 * 128))
        if x.data_ptr() != self.x.data_ptr():
            self.x[:n].copy_(x)
        if n < m:
            self.x[n:m].zero_()
        if target is not None and not (train and n == B):
            raise ValueError("a fused target needs a full training batch")
        if not self.fused:
            self._target_fused = False
            return self._forward_layers(n, m, train)
        st = self.lib.lcg_mlp_forward(self._stream(), _p(self.x), self.nin, m, n, _p(self.W[0]),
                                      _p(self.b[0]), self.depth, self.nout, self._fw_w,
                                      self._fw_b, _p(self.out), self._fw_z if train else None,
                                      self._fw_yt if train else None, B, _p(target),
                                      _p(self.G[self.depth]), _p(self.Gt[self.depth]),
                                      _p(self.loss_rows), _p(self.err))
        self._ok(st, "lcg_mlp_forward")
        self._target_fused = target is not None
        return self.out[:n]

    def _forward_layers(self, n, m, train):
        """One launch per layer (lcg_mlp_input, lcg_mlp_gemm)."""
        B, w = self.B, self.width
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

    def backward(self, target=None, sync=True):
        """Gradients of the mean squared error of the last forward (a full
        training batch) against target [B, nout], or against the target the
        forward already took. Returns the loss (sync=True) or None (no host
        synchronisation)."""
        B, w, L = self.B, self.width, self.depth
        if not self._target_fused:
            if target is None:
                raise ValueError("backward needs the target")
            st = self.lib.lcg_mlp_mse_grad(self._stream(), _p(self.out), _p(target), B, self.nout,
                                           B, B, _p(self.G[L]), _p(self.Gt[L]),
                                           _p(self.loss_rows))
            self._ok(st, "lcg_mlp_mse_grad")
        self._target_fused = False
        if self.fused:
            st = self.lib.lcg_mlp_backward_data(self._stream(), B, L, self.nout, _p(self.G[L]),
                                                self._bw_wt, self._bw_z, self._bw_g, self._bw_gt,
                                                B, _p(self.err))
            self._ok(st, "lcg_mlp_backward_data")
            for l in range(L, 0, -1):
                self._gemm(EPI_F32, self.Gt[l].shape[0], w, B, self.Gt[l], self.Yt[l - 1],
                           out=self.dW[l], mvalid=self.nout if l == L else w)
                self._colsum(self.G[l], self.nout if l == L else w, self.db[l])
        else:
            self._backward_layers()
        st = self.lib.lcg_mlp_input_grad(self._stream(), _p(self.G[0]), _p(self.x), self.nin, B,
                                         w, B, _p(self.dW[0]))
        self._ok(st, "lcg_mlp_input_grad")
        self._colsum(self.G[0], w, self.db[0])
        if sync:
            return float(self.loss_rows.sum().item()) / (B * self.nout)
        return None

    def _backward_layers(self):
        """The backward chain one GEMM per launch (lcg_mlp_gemm)."""
        B, w, L = self.B, self.width, self.depth
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

    # -- graph-captured training -------------------------------------------------
    def set_schedule(self, lr_max, lr_min=None, total_steps=0, beta1=0.9, beta2=0.999, eps=1e-8):
        """The device-side Adam schedule of graph_step: cosine from lr_max to
        lr_min over total_steps (constant lr_max when total_steps is 0);
        restarts the step count and the moments' bias corrections."""
        torch = self.torch
        lo = lr_max if lr_min is None else lr_min
        self.sched.copy_(torch.tensor([lr_max, lo, float(total_steps), beta1, beta2, eps],
                                      dtype=torch.float32))
        self.step_dev.zero_()

    def _train_ops(self):
        torch = self.torch
        self.forward(self.x, train=True, target=self.tgt)
        self.backward(sync=False)
        n, w, m1, m2, g, wb, wt = self._adam
        st = self.lib.lcg_mlp_adam_all(self._stream(), n, w, m1, m2, g, self._adam_rows,
                                       self._adam_cols, wb, wt, _p(self.sched),
                                       _p(self.step_dev))
        self._ok(st, "lcg_mlp_adam_all")
        self.step_dev.add_(1)
        self.loss_acc.add_(self.loss_rows.sum(dtype=torch.float64))

    def graph_step(self):
        """One training step on the batch in self.x / self.tgt: fused forward
        with the loss gradient, backward chain, weight and bias gradients,
        Adam on the device schedule (set_schedule), the step count advanced
        and the batch loss added to loss_acc; no host synchronisation. The
        first call runs eagerly and captures the same launches as a CUDA
        graph, which later calls replay."""
        torch = self.torch
        if self._graph is not None:
            self._graph.replay()
            return
        self._train_ops()
        s = torch.cuda.Stream(device=self.dev)
        s.wait_stream(torch.cuda.current_stream(self.dev))
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                self._train_ops()
        torch.cuda.current_stream(self.dev).wait_stream(s)
        self._graph = g

    def take_loss(self):
        """The mean squared error summed over the graph steps since the last
        call (divided by batch x nout per step), and resets the sum."""
        v = float(self.loss_acc.item()) / (self.B * self.nout)
        self.loss_acc.zero_()
        return v

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
