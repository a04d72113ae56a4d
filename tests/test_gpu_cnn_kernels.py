"""GPU checks of the learned-initialiser kernels: the tcgen05 BF16 GEMM against an
FP64 product of the same BF16-rounded operands, and every layer kernel against
torch's FP32/FP64 CPU implementation of the same op (the layers of the
reference's CNN2d, core/ml/cnn.py and core/ml/blocks.py)."""
import pytest
import torch
import torch.nn.functional as F

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = a.double().cpu()
    b = b.double().cpu()
    return float((a - b).norm() / max(b.norm(), 1e-30))


def _bf(x):
    return x.to(torch.bfloat16)


@pytest.mark.parametrize(
    "M,N,K,splits",
    [(128, 32, 64, 1), (200, 40, 72, 1), (1000, 130, 520, 1), (64, 1024, 576, 1), (777, 64, 4104, 3),
     (4096, 36, 288, 1), (96, 300, 8192, 8)],
)
def test_gemm_fp32_out(cuda_device, M, N, K, splits):
    from quantem_b200.core.ml import kernels as kk

    g = torch.Generator().manual_seed(M * 7 + N)
    A = _bf(torch.randn(M, K, generator=g))
    B = _bf(torch.randn(N, K, generator=g))
    bias = torch.randn(N, generator=g)
    ref = A.double() @ B.double().T + bias.double()
    C = torch.full((M, N), float("nan"), device=cuda_device)
    st = torch.zeros(1, dtype=torch.int32, device=cuda_device)
    kk.gemm(A.to(cuda_device), B.to(cuda_device), C, bias=bias.to(cuda_device), splits=splits, status=st)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    assert _rel(C, ref) < 1e-5


def test_gemm_bf16_relu_strided(cuda_device):
    """BF16 + ReLU epilogue into a column slice of a wider buffer; A and B are
    strided row views (leading dimensions larger than K)."""
    from quantem_b200.core.ml import kernels as kk

    g = torch.Generator().manual_seed(5)
    M, N, K = 300, 64, 200
    Abig = _bf(torch.randn(M, 256, generator=g))
    Bbig = _bf(torch.randn(N, 208, generator=g))
    bias = torch.randn(N, generator=g)
    ref = torch.relu(Abig[:, :K].double() @ Bbig[:, :K].double().T + bias.double())
    out = torch.zeros(M, 160, dtype=torch.bfloat16, device=cuda_device)
    Ad, Bd = Abig.to(cuda_device), Bbig.to(cuda_device)
    kk.gemm(Ad[:, :K], Bd[:, :K], out[:, 32:96], bias=bias.to(cuda_device), relu=True)
    torch.cuda.synchronize()
    got = out[:, 32:96].float()
    assert _rel(got, ref) < 8e-3  # BF16 output rounding
    assert float(out[:, :32].abs().max()) == 0.0 and float(out[:, 96:].abs().max()) == 0.0


def test_gemm_rejects_bad_arguments(cuda_device):
    from quantem_b200.core.ml import kernels as kk

    A = torch.zeros(16, 30, dtype=torch.bfloat16, device=cuda_device)  # leading dimension 30: not a multiple of 8
    B = torch.zeros(16, 30, dtype=torch.bfloat16, device=cuda_device)
    C = torch.zeros(16, 16, device=cuda_device)
    with pytest.raises(RuntimeError, match="multiple of 8"):
        kk.gemm(A, B, C)


def _nhwc(x):  # (B, C, H, W) -> (B*H*W, C)
    b, c, h, w = x.shape
    return x.permute(0, 2, 3, 1).reshape(b * h * w, c).contiguous()


def _nchw(m, b, h, w):
    return m.reshape(b, h, w, -1).permute(0, 3, 1, 2).contiguous()


def test_conv3x3_circular_forward_and_adjoint(cuda_device):
    """im2col + GEMM = nn.Conv2d(3x3, padding 1, circular); col2im is the exact adjoint."""
    from quantem_b200.core.ml import kernels as kk

    g = torch.Generator().manual_seed(11)
    Bn, Ci, Co, H, W = 2, 16, 24, 8, 12
    x = _bf(torch.randn(Bn, Ci, H, W, generator=g)).float()
    w = _bf(torch.randn(Co, Ci, 3, 3, generator=g) * 0.2).float()
    b = torch.randn(Co, generator=g)
    ref = F.conv2d(F.pad(x.double(), (1, 1, 1, 1), mode="circular"), w.double(), b.double())
    xd = _nhwc(x).to(torch.bfloat16).to(cuda_device)
    col = torch.empty(Bn * H * W, 9 * Ci, dtype=torch.bfloat16, device=cuda_device)
    kk.im2col3x3(xd, Bn, H, W, col)
    wk = _bf(w.permute(0, 2, 3, 1).reshape(Co, 9 * Ci)).to(cuda_device)  # (co, ky, kx, ci)
    y = torch.empty(Bn * H * W, Co, device=cuda_device)
    kk.gemm(col, wk, y, bias=b.to(cuda_device))
    assert _rel(_nchw(y.cpu(), Bn, H, W), ref) < 1e-5
    # adjoint: <im2col(x), d> == <x, col2im(d)>
    d = torch.randn(Bn * H * W, 9 * Ci, generator=g).to(cuda_device)
    dx = torch.empty(Bn * H * W, Ci, device=cuda_device)
    kk.col2im3x3(d, Bn, H, W, Ci, dx)
    lhs = float((col.double() * d.double()).sum())
    rhs = float((xd.double() * dx.double()).sum())
    assert abs(lhs - rhs) <= 1e-9 * max(1.0, abs(lhs)) + 1e-3


def test_conv_transpose_forward_and_adjoint(cuda_device):
    """GEMM + convT_gather = nn.ConvTranspose2d(3, stride 2, padding 1, output_padding 1)."""
    from quantem_b200.core.ml import kernels as kk

    g = torch.Generator().manual_seed(12)
    Bn, Ci, Co, H, W = 2, 16, 8, 5, 6
    x = _bf(torch.randn(Bn, Ci, H, W, generator=g)).float()
    w = _bf(torch.randn(Ci, Co, 3, 3, generator=g) * 0.3).float()  # torch layout (in, out, kh, kw)
    b = torch.randn(Co, generator=g)
    ref = F.conv_transpose2d(x.double(), w.double(), b.double(), stride=2, padding=1, output_padding=1)
    xd = _nhwc(x).to(torch.bfloat16).to(cuda_device)
    wk = _bf(w.permute(2, 3, 1, 0).reshape(9 * Co, Ci)).to(cuda_device)  # (ky, kx, co) x ci
    colT = torch.empty(Bn * H * W, 9 * Co, device=cuda_device)
    kk.gemm(xd, wk, colT)
    out = torch.empty(Bn * 4 * H * W, Co, dtype=torch.bfloat16, device=cuda_device)
    kk.convT_gather(colT, Bn, H, W, Co, b.to(cuda_device), out)
    assert _rel(_nchw(out.float().cpu(), Bn, 2 * H, 2 * W), ref) < 8e-3
    # adjoint of the gather: <gather(c), d> == <c, convT_im2col(d)> (gather output rounded to BF16)
    c = _bf(torch.randn(Bn * H * W, 9 * Co, generator=g)).float().to(cuda_device)
    gout = torch.empty(Bn * 4 * H * W, Co, dtype=torch.bfloat16, device=cuda_device)
    kk.convT_gather(c, Bn, H, W, Co, None, gout)
    d = _bf(torch.randn(Bn * 4 * H * W, Co, generator=g)).float().to(cuda_device)
    dc = torch.empty(Bn * H * W, 9 * Co, dtype=torch.bfloat16, device=cuda_device)
    kk.convT_im2col(d, Bn, H, W, Co, dc)
    lhs = float((gout.double() * d.double()).sum())
    rhs = float((c.double() * dc.double()).sum())
    assert abs(lhs - rhs) <= 5e-3 * float(gout.double().norm() * d.double().norm())


def test_batchnorm_relu_forward_backward(cuda_device):
    from quantem_b200.core.ml import kernels as kk

    g = torch.Generator().manual_seed(13)
    R, C = 4096, 48
    x = torch.relu(torch.randn(R, C, generator=g) * 2 + 0.3)
    gamma = torch.rand(C, generator=g) + 0.5
    beta = torch.randn(C, generator=g)
    dy = torch.randn(R, C, generator=g)
    xr = x.double().requires_grad_(True)
    gr = gamma.double().requires_grad_(True)
    br = beta.double().requires_grad_(True)
    rm, rv = torch.zeros(C, dtype=torch.float64), torch.ones(C, dtype=torch.float64)
    yr = F.batch_norm(xr, rm, rv, gr, br, training=True, momentum=0.1, eps=1e-5)
    yr.backward(dy.double())
    dev = cuda_device
    xd, gd, bd = x.to(dev), gamma.to(dev), beta.to(dev)
    rmd, rvd = torch.zeros(C, device=dev), torch.ones(C, device=dev)
    mean, rstd = torch.empty(C, device=dev), torch.empty(C, device=dev)
    work = torch.empty(64 * C, dtype=torch.float64, device=dev)
    y = torch.empty(R, C, dtype=torch.bfloat16, device=dev)
    kk.bn_forward(xd, gd, bd, rmd, rvd, 0.1, 1e-5, True, mean, rstd, work, y)
    assert _rel(y.float(), yr.detach()) < 8e-3
    assert _rel(rmd, rm) < 1e-6 and _rel(rvd, rv) < 1e-6
    dg, db = torch.empty(C, device=dev), torch.empty(C, device=dev)
    dz = torch.empty(R, C, device=dev)
    kk.bn_backward(dy.to(dev), xd, gd, mean, rstd, True, True, dg, db, work, dz32=dz)
    ref_dz = xr.grad * (x.double() > 0)
    assert _rel(dz, ref_dz) < 1e-5
    assert _rel(dg, gr.grad) < 1e-5 and _rel(db, br.grad) < 1e-5
    s = torch.empty(C, device=dev)
    kk.colsum(dz, s, work)
    assert _rel(s, ref_dz.sum(0)) < 1e-5


def test_maxpool_transpose_cast_mse(cuda_device):
    from quantem_b200.core.ml import kernels as kk

    g = torch.Generator().manual_seed(14)
    Bn, C, H, W = 2, 8, 6, 10
    x = _bf(torch.randn(Bn, C, H, W, generator=g)).float()
    xr = x.clone().requires_grad_(True)
    ref = F.max_pool2d(xr, 2, 2)
    dref = torch.randn_like(ref)
    ref.backward(dref)
    dev = cuda_device
    xd = _nhwc(x).to(torch.bfloat16).to(dev)
    out = torch.empty(Bn * H * W // 4, C, dtype=torch.bfloat16, device=dev)
    arg = torch.empty(Bn * H * W // 4, C, dtype=torch.uint8, device=dev)
    kk.maxpool2(xd, Bn, H, W, out, arg)
    assert torch.equal(_nchw(out.float().cpu(), Bn, H // 2, W // 2), ref.detach())
    din = torch.empty(Bn * H * W, C, device=dev)
    kk.maxpool2_backward(_nhwc(dref).to(dev), arg, Bn, H, W, din)
    assert torch.equal(_nchw(din.cpu(), Bn, H, W), xr.grad)
    # batched NCHW -> channels-last transpose and back
    t = torch.randn(3, 40, 70, generator=g).to(dev)
    tt = torch.empty(3, 70, 40, dtype=torch.bfloat16, device=dev)
    kk.transpose(t, tt)
    assert _rel(tt.float(), t.transpose(1, 2)) < 5e-3
    back = torch.empty(3, 40, 70, device=dev)
    kk.transpose(tt, back)
    assert torch.equal(back, tt.float().transpose(1, 2))
    c16 = torch.empty(3, 40, 70, dtype=torch.bfloat16, device=dev)
    kk.cast_bf16(t, c16)
    assert torch.equal(c16, t.to(torch.bfloat16))
    p, q = torch.randn(1000, generator=g), torch.randn(1000, generator=g)
    loss = torch.empty(1, device=dev)
    work = torch.empty(296, dtype=torch.float64, device=dev)
    dp = torch.empty(1000, device=dev)
    kk.mse(p.to(dev), q.to(dev), loss, work, dpred32=dp)
    assert abs(float(loss.item()) - float(((p - q) ** 2).mean())) < 1e-6
    assert _rel(dp, 2 * (p - q) / 1000) < 1e-6
