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
