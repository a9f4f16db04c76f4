"""The surrogate network's kernels on the GPU.

  * lcg_mlp_gemm against a torch FP32 product of the same BF16 operands:
    FP32 outputs within 1e-5 of the largest magnitude (summation order),
    BF16 outputs within one BF16 rounding (8e-3 relative);
  * the FP32 input layer and the PCA chi**2 head against numpy;
  * the network's weight and bias gradients against the FP64 oracle
    (oracle/mlp_oracle.py), which rounds to BF16 where the kernels store
    BF16: relative Frobenius error <= 2e-2 per layer;
  * training on the tensor cores reduces the loss.
"""
import ctypes as C
import os
import sys

import numpy as np
import pytest

from lcurve_re_b200 import abi

pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                "oracle"))


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


@pytest.fixture(scope="module")
def lib():
    from lcurve_re_b200.engine import load_library
    return load_library()


def _gemm(lib, torch, epi, a, b, bias=None, z=None, y=None, yt=None, out=None, mvalid=None,
          ldt=0):
    m, k = a.shape
    n = b.shape[0]
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = lib.lcg_mlp_gemm(C.c_void_p(torch.cuda.current_stream().cuda_stream), epi, m, n, k,
                          _p(a), _p(b), _p(bias), _p(z), _p(y), _p(yt), _p(out),
                          m if mvalid is None else mvalid, ldt, _p(err))
    torch.cuda.synchronize()
    assert st == abi.OK and int(err.item()) == 0
    return st


@pytest.mark.parametrize("m,n,k", [(128, 64, 64), (256, 256, 128), (384, 512, 320),
                                   (128, 256, 4096)])
def test_gemm_f32_and_linear(lib, m, n, k):
    import torch
    g = torch.Generator(device="cuda").manual_seed(m + n + k)
    a = torch.randn(m, k, device="cuda", generator=g).to(torch.bfloat16)
    b = torch.randn(n, k, device="cuda", generator=g).to(torch.bfloat16)
    ref = a.float() @ b.float().T
    out = torch.full((m, n), 7.0, device="cuda")
    _gemm(lib, torch, 3, a, b, out=out)
    scale = ref.abs().max().item()
    assert (out - ref).abs().max().item() <= 1e-5 * scale
    bias = torch.randn(n, device="cuda", generator=g)
    out2 = torch.full((m, n), 7.0, device="cuda")
    _gemm(lib, torch, 1, a, b, bias=bias, out=out2, mvalid=m - 5)
    assert (out2[:m - 5] - (ref + bias)[:m - 5]).abs().max().item() <= 1e-5 * scale
    assert torch.all(out2[m - 5:] == 7.0)


def _bf_close(x, ref):
    x, ref = x.float(), ref.float()
    return (x - ref).abs().max().item() <= 8e-3 * ref.abs().max().item() + 1e-6


def test_gemm_gelu_and_dgelu(lib):
    import torch
    m, n, k = 256, 256, 192
    g = torch.Generator(device="cuda").manual_seed(5)
    a = (0.3 * torch.randn(m, k, device="cuda", generator=g)).to(torch.bfloat16)
    b = (0.3 * torch.randn(n, k, device="cuda", generator=g)).to(torch.bfloat16)
    bias = 0.1 * torch.randn(n, device="cuda", generator=g)
    zr = a.float() @ b.float().T + bias
    z = torch.zeros(m, n, dtype=torch.bfloat16, device="cuda")
    y = torch.zeros_like(z)
    yt = torch.zeros(n, m, dtype=torch.bfloat16, device="cuda")
    _gemm(lib, torch, 0, a, b, bias=bias, z=z, y=y, yt=yt, ldt=m)
    gelu = torch.nn.functional.gelu
    assert _bf_close(z, zr)
    assert _bf_close(y, gelu(zr))
    assert torch.equal(yt, y.T.contiguous())
    # backward epilogue: D * GELU'(z) with z read back
    d = (a.float() @ b.float().T)
    zz = z.float().requires_grad_(True)
    gelu(zz).backward(torch.ones_like(zz))
    gr = d * zz.grad
    g2 = torch.zeros_like(z)
    g2t = torch.zeros_like(yt)
    _gemm(lib, torch, 2, a, b, z=z, y=g2, yt=g2t, ldt=m)
    assert _bf_close(g2, gr)
    assert torch.equal(g2t, g2.T.contiguous())


def test_input_layer_and_pca_chisq(lib):
    import torch
    m, kin, n = 256, 9, 256
    x = torch.rand(m, kin, device="cuda") * 2 - 1
    w = torch.randn(n, kin, device="cuda")
    b = torch.randn(n, device="cuda")
    z = torch.zeros(m, n, dtype=torch.bfloat16, device="cuda")
    y = torch.zeros_like(z)
    yt = torch.zeros(n, m, dtype=torch.bfloat16, device="cuda")
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert lib.lcg_mlp_input(s, _p(x), kin, _p(w), _p(b), m, n, m - 3, _p(z), _p(y), _p(yt),
                             m) == abi.OK
    zr = x @ w.T + b
    zr[m - 3:] = 0
    assert _bf_close(z, zr) and _bf_close(y, torch.nn.functional.gelu(zr))
    assert torch.equal(yt, y.T.contiguous())
    # chi**2 head
    rows, nc, npts = 7, 64, 500
    coef = torch.randn(rows, nc, device="cuda")
    basis = 1e-3 * torch.randn(nc, npts, device="cuda")
    mean = 1 + 0.1 * torch.rand(npts, device="cuda")
    flux = (1.3 * mean + 1e-3 * torch.randn(npts, device="cuda")).double()
    ferr = torch.full((npts,), 1.5e-3, dtype=torch.float64, device="cuda")
    wgt = torch.ones(npts, dtype=torch.float64, device="cuda")
    wgt[3] = 0.0
    chi = torch.zeros(rows, dtype=torch.float64, device="cuda")
    sc = torch.zeros_like(chi)
    assert lib.lcg_mlp_pca_chisq(s, _p(coef), rows, nc, _p(basis), _p(mean), npts, _p(flux),
                                 _p(ferr), _p(wgt), None, None, _p(chi), _p(sc)) == abi.OK
    f = (mean[None, :].double() + coef.double() @ basis.double())
    wv = (wgt / ferr ** 2)[None, :]
    s_ref = (wv * flux * f).sum(1) / (wv * f * f).sum(1)
    chi_ref = (wgt[None, :] * ((flux[None, :] - s_ref[:, None] * f) / ferr) ** 2).sum(1)
    assert torch.allclose(sc, s_ref, rtol=1e-6)
    assert torch.allclose(chi, chi_ref, rtol=1e-4)
    # anchored: an exact curve times the surrogate's ratio between two points
    coef_x = torch.randn(rows, nc, device="cuda")
    anchor = (1 + 0.05 * torch.rand(rows, npts, device="cuda")).double()
    assert lib.lcg_mlp_pca_chisq(s, _p(coef), rows, nc, _p(basis), _p(mean), npts, _p(flux),
                                 _p(ferr), _p(wgt), _p(coef_x), _p(anchor), _p(chi),
                                 _p(sc)) == abi.OK
    g = (mean[None, :].double() + coef_x.double() @ basis.double())
    f = anchor * (f / g)
    s_ref = (wv * flux * f).sum(1) / (wv * f * f).sum(1)
    chi_ref = (wgt[None, :] * ((flux[None, :] - s_ref[:, None] * f) / ferr) ** 2).sum(1)
    assert torch.allclose(sc, s_ref, rtol=1e-5)
    assert torch.allclose(chi, chi_ref, rtol=1e-3)


def test_gradients_match_the_oracle():
    import torch
    import mlp_oracle as O
    from lcurve_re_b200.mlp import MLP
    net = MLP(batch=256, seed=3)
    rng = np.random.default_rng(4)
    x = rng.uniform(-1, 1, (256, 9))
    t = rng.standard_normal((256, 64)) * 0.5
    net.forward(torch.as_tensor(x, dtype=torch.float32, device="cuda"), train=True)
    loss = net.backward(torch.as_tensor(t, dtype=torch.float32, device="cuda"))
    torch.cuda.synchronize()
    net.check()
    W = [w.cpu().numpy().astype(np.float64) for w in net.W]
    b = [v.cpu().numpy().astype(np.float64) for v in net.b]
    lo, dW, db, out = O.backward(W, b, x.astype(np.float32).astype(np.float64), t)
    assert abs(loss - lo) <= 1e-2 * lo
    np.testing.assert_allclose(net.out.cpu().numpy(), out, rtol=0, atol=2e-2 * np.abs(out).max())
    for l in range(len(W)):
        g = net.dW[l][:W[l].shape[0]].cpu().numpy()
        rel = np.linalg.norm(g - dW[l]) / np.linalg.norm(dW[l])
        assert rel <= 2e-2, (l, rel)
        relb = np.linalg.norm(net.db[l].cpu().numpy() - db[l]) / np.linalg.norm(db[l])
        assert relb <= 2e-2, (l, relb)


def test_training_reduces_the_loss():
    import torch
    from lcurve_re_b200.mlp import MLP
    net = MLP(batch=1024, nout=64, seed=0)
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.rand(1024, 9, device="cuda", generator=g) * 2 - 1
    proj = torch.randn(9, 64, device="cuda", generator=g)
    t = torch.sin(2 * x @ proj).contiguous()
    losses = []
    for it in range(300):
        net.forward(x, train=True)
        losses.append(net.backward(t))
        net.step(1e-3)
    net.check()
    assert losses[-1] < 0.1 * losses[0], (losses[0], losses[-1])


def test_inference_on_the_rows_present_matches_the_full_batch():
    """Inference runs only ceil(n / 128) x 128 rows; the outputs of those rows
    equal a full-batch pass (FP32 sums of the same BF16 products)."""
    import torch
    from lcurve_re_b200.mlp import MLP
    net = MLP(nin=9, nout=64, batch=1024, device="cuda", seed=3)
    x = torch.rand(1024, 9, device="cuda")
    full = net.forward(x).clone()
    for n in (1, 130, 512):
        part = net.forward(x[:n]).clone()
        torch.testing.assert_close(part, full[:n], rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("m,n,k,dtype", [(300, 200, 1000, "float64"), (1000, 1000, 5000, "float64"),
                                         (777, 64, 130, "float32"), (256, 192, 20000, "float64")])
def test_split_bf16_gemm_reaches_fp32_accuracy(m, n, k, dtype):
    """gemm_bf16x3 (three BF16 products on lcg_mlp_gemm, K blocks of 8192
    summed in FP64) against the FP64 product: every entry within 3e-5 of the
    largest |a| |b|^T entry, which one BF16 product (about 4e-3) misses by
    two orders of magnitude."""
    import torch
    from lcurve_re_b200.mlp import gemm_bf16x3
    g = torch.Generator(device="cuda").manual_seed(m + n + k)
    dt = getattr(torch, dtype)
    a = torch.randn(m, k, device="cuda", generator=g, dtype=torch.float64).to(dt)
    b = torch.randn(n, k, device="cuda", generator=g, dtype=torch.float64).to(dt)
    ref = a.double() @ b.double().T
    bound = (a.double().abs() @ b.double().abs().T).max().item()
    out = gemm_bf16x3(a, b)
    torch.cuda.synchronize()
    assert out.shape == (m, n) and out.dtype == torch.float64
    err = (out - ref).abs().max().item() / bound
    assert err <= 3e-5, err
    one = (a.to(torch.bfloat16).double() @ b.to(torch.bfloat16).double().T - ref).abs().max()
    assert one.item() / bound > 100 * err


def test_pca_on_the_tensor_cores_matches_fp64():
    """Surrogate.fit_pca (Gram matrix, coefficients and reconstruction on
    gemm_bf16x3) against the same PCA in FP64 torch on curves of 64 modes
    (amplitudes 1e-2 .. 1e-4) plus a 16-mode tail (1e-5) and noise, so the
    retained subspace is well determined: its principal angles' cosines
    >= 1 - 1e-5 (the Gram matrix carries FP32 rounding, about 1e-7 of its
    largest eigenvalue, against a gap of 1e-4 of it at the cut: angles up to
    ~1e-3), the reconstruction residual's maximum within 10% of the FP64 one,
    and the coefficients within 1e-5 of their largest magnitude."""
    import torch
    from lcurve_re_b200.surrogate import Surrogate
    rng = np.random.default_rng(5)
    n, npts = 20000, 1000
    amp = np.r_[np.logspace(-2, -4, 64), np.logspace(-5, -5.5, 16)]
    modes = rng.standard_normal((80, npts)) * amp[:, None]
    curves = 1.0 + rng.standard_normal((n, 80)) @ modes + 1e-7 * rng.standard_normal((n, npts))
    sur = Surrogate(batch=256)
    err, target = sur.fit_pca(curves)
    y = torch.as_tensor(curves, device="cuda")
    yc = y - y.mean(0)
    ev, V = torch.linalg.eigh(yc.T @ yc / n)
    basis = V[:, torch.argsort(ev, descending=True)[:sur.ncoef]].T
    ref_err = float((yc - (yc @ basis.T) @ basis).abs().max())
    cos = torch.linalg.svdvals(sur.basis @ basis.T)
    assert float(cos.min()) >= 1 - 1e-5, float(cos.min())
    assert abs(err - ref_err) <= 0.1 * ref_err, (err, ref_err)
    coef_ref = (yc @ sur.basis.T) / sur.cscale
    assert float((target - coef_ref).abs().max()) <= 1e-5 * float(coef_ref.abs().max())


def _bits_close(a, b, what):
    """BF16 tensors equal up to one rounding step of BF16 (the one-launch
    chain and the per-layer kernels may round a product sum differently in
    the last FP32 bit)."""
    import torch
    a, b = a.float(), b.float()
    tol = 2 ** -7 * torch.maximum(a.abs(), b.abs()) + 1e-30
    bad = int(((a - b).abs() > tol).sum())
    assert bad == 0, (what, bad)


@pytest.mark.parametrize("n", [1, 130, 512, 1024])
def test_fused_forward_matches_the_layer_by_layer_kernels(n):
    """lcg_mlp_forward (all layers in one launch) against lcg_mlp_input +
    lcg_mlp_gemm per layer on the same weights: inference outputs within
    1e-5 relative, and in training the stored pre-activations and
    transposed activations of every layer within one BF16 rounding."""
    import torch
    from lcurve_re_b200.mlp import MLP
    net = MLP(nin=9, nout=64, batch=1024, seed=11)
    for l in range(1, net.depth + 1):  # non-zero biases
        net.b[l].copy_(0.1 * torch.randn_like(net.b[l]))
    x = torch.rand(n, 9, device="cuda") * 2 - 1
    fused = net.forward(x).clone()
    net.fused = False
    ref = net.forward(x).clone()
    torch.testing.assert_close(fused, ref, rtol=1e-5, atol=1e-5 * float(ref.abs().max()))
    if n == 1024:
        net.forward(x, train=True)
        ref_z = [z.clone() for z in net.Z]
        ref_yt = [y.clone() for y in net.Yt]
        ref_out = net.out.clone()
        net.fused = True
        net.forward(x, train=True)
        for l in range(net.depth):
            _bits_close(net.Z[l], ref_z[l], ("z", l))
            _bits_close(net.Yt[l], ref_yt[l], ("yt", l))
        torch.testing.assert_close(net.out, ref_out, rtol=1e-5,
                                   atol=1e-5 * float(ref_out.abs().max()))


def test_fused_backward_matches_the_layer_by_layer_kernels():
    """Forward with the fused loss gradient + lcg_mlp_backward_data against
    lcg_mlp_mse_grad + one GEMM per layer: every layer's gradient (and its
    transpose) within one BF16 rounding, weight and bias gradients within
    1e-3 of their largest entry, the same loss to 1e-6."""
    import torch
    from lcurve_re_b200.mlp import MLP
    net = MLP(nin=9, nout=64, batch=512, seed=12)
    x = torch.rand(512, 9, device="cuda") * 2 - 1
    t = torch.randn(512, 64, device="cuda").contiguous()
    net.fused = False
    net.forward(x, train=True)
    loss_ref = net.backward(t)
    G = [g.clone() for g in net.G]
    Gt = [g.clone() for g in net.Gt]
    dW = [d.clone() for d in net.dW]
    db = [d.clone() for d in net.db]
    net.fused = True
    net.x.copy_(x)
    net.tgt.copy_(t)
    net.forward(net.x, train=True, target=net.tgt)
    loss = net.backward()
    net.check()
    assert abs(loss - loss_ref) <= 1e-6 * loss_ref
    for l in range(net.depth + 1):
        _bits_close(net.G[l], G[l], ("g", l))
        if l >= 1:
            _bits_close(net.Gt[l], Gt[l], ("gt", l))
        tol = 1e-3 * float(dW[l].abs().max())
        assert float((net.dW[l] - dW[l]).abs().max()) <= tol, ("dW", l)
        assert float((net.db[l] - db[l]).abs().max()) <= 1e-3 * float(db[l].abs().max()), l


def test_graph_training_steps_follow_the_eager_steps():
    """graph_step (one captured graph: fused chains, weight gradients and
    the one-launch Adam on the device-side cosine schedule) against eager
    forward/backward/step with the same learning rates: weights within 1e-4
    relative after 20 steps, and the loss falls over 300 steps."""
    import torch
    from lcurve_re_b200.mlp import MLP
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.rand(1024, 9, device="cuda", generator=g) * 2 - 1
    proj = torch.randn(9, 64, device="cuda", generator=g)
    t = torch.sin(2 * x @ proj).contiguous()
    a, b = MLP(batch=1024, seed=5), MLP(batch=1024, seed=5)
    total, lr, lr_min = 20, 2e-3, 2e-4
    b.set_schedule(lr, lr_min, total)
    for k in range(total):
        a.forward(x, train=True)
        a.backward(t)
        a.step(lr_min + 0.5 * (lr - lr_min) * (1 + np.cos(np.pi * k / total)))
        b.x.copy_(x)
        b.tgt.copy_(t)
        b.graph_step()
    torch.cuda.synchronize()
    a.check()
    b.check()
    assert int(b.step_dev.item()) == total
    for l in range(a.depth + 1):
        rel = float((a.W[l] - b.W[l]).norm() / a.W[l].norm())
        assert rel <= 1e-4, (l, rel)
    b.set_schedule(1e-3)
    first = None
    for k in range(300):
        b.graph_step()
        if k == 0:
            first = b.take_loss()
    b.take_loss()
    b.graph_step()
    last = b.take_loss()
    assert last < 0.1 * first, (first, last)
