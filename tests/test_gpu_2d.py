"""2-D transforms and transforms along a middle axis (column kernel) through the C ABI and the
torch layer, against FP64 numpy.

Tolerances: a 2-D transform is a row pass and a column pass, each within the 1-D fp32 error,
so the gate is rel L2 <= 2e-6 per matrix (the long-transform tolerance); a single transform
along a middle axis is gated like a 1-D transform (rel L2 <= 1e-6 per transform).
Shapes follow the reference's planned 2-D / range-Doppler cases (square 256^2..2048^2 and
rectangular 1024x128) plus the envelope edges (ny = 32 and 4096, nx up to 65536)."""
import numpy as np
import pytest

import oracle.fft_oracle as O

pytestmark = pytest.mark.gpu


def _rel_mats(got, ref):
    got = got.reshape(-1, got.shape[-2] * got.shape[-1])
    ref = ref.reshape(-1, ref.shape[-2] * ref.shape[-1])
    return O.rel_l2_rows(got, ref)


def _cplx(shape, seed, cuda):
    import torch
    g = torch.Generator(device=cuda).manual_seed(seed)
    return torch.randn(*shape, dtype=torch.complex64, device=cuda, generator=g)


@pytest.mark.parametrize("ny,nx", [(32, 64), (256, 256), (512, 512), (1024, 128), (128, 1024),
                                   (64, 4096), (4096, 32), (2048, 2048), (32, 65536)])
@pytest.mark.parametrize("direction", [-1, 1])
def test_2d_matches_fp64(plan, cuda, ny, nx, direction):
    import torch
    batch = 2 if ny * nx <= (1 << 20) else 1
    x = _cplx((batch, ny, nx), 1000 + ny + nx, cuda)
    y = torch.empty_like(x)
    scale = 1.0 if direction < 0 else 1.0 / (ny * nx)
    assert plan.exec_c2c_2d(x.data_ptr(), y.data_ptr(), ny, nx, batch, direction, scale, 0) == 0
    torch.cuda.synchronize()
    xd = x.cpu().numpy().astype(np.complex128)
    ref = np.fft.fft2(xd) if direction < 0 else np.fft.ifft2(xd)
    assert _rel_mats(y.cpu().numpy(), ref) <= 2e-6


def test_2d_in_place_and_round_trip(plan, cuda):
    import torch
    ny, nx, batch = 512, 256, 3
    x = _cplx((batch, ny, nx), 7, cuda)
    y = torch.empty_like(x)
    assert plan.exec_c2c_2d(x.data_ptr(), y.data_ptr(), ny, nx, batch, -1, 1.0, 0) == 0
    z = x.clone()
    assert plan.exec_c2c_2d(z.data_ptr(), z.data_ptr(), ny, nx, batch, -1, 1.0, 0) == 0
    torch.cuda.synchronize()
    assert torch.equal(y, z)
    assert plan.exec_c2c_2d(y.data_ptr(), z.data_ptr(), ny, nx, batch, 1, 1.0 / (ny * nx), 0) == 0
    torch.cuda.synchronize()
    assert (torch.linalg.vector_norm(z - x) / torch.linalg.vector_norm(x)).item() <= 4e-6


@pytest.mark.parametrize("n", [32, 256, 4096])
@pytest.mark.parametrize("outer,inner", [(1, 3), (2, 16), (3, 130), (1, 1024)])
def test_axis_matches_fp64(plan, cuda, n, outer, inner):
    import torch
    x = _cplx((outer, n, inner), 31 + n + inner, cuda)
    y = torch.empty_like(x)
    assert plan.exec_c2c_axis(x.data_ptr(), y.data_ptr(), n, outer, inner, -1, 1.0, 0) == 0
    torch.cuda.synchronize()
    ref = np.fft.fft(x.cpu().numpy().astype(np.complex128), axis=1)
    got = np.moveaxis(y.cpu().numpy(), 1, -1).reshape(-1, n)
    assert O.rel_l2_rows(got, np.moveaxis(ref, 1, -1).reshape(-1, n)) <= 1e-6
    z = x.clone()   # in place, inverse with scale: back to the input
    assert plan.exec_c2c_axis(z.data_ptr(), z.data_ptr(), n, outer, inner, -1, 1.0, 0) == 0
    assert plan.exec_c2c_axis(z.data_ptr(), z.data_ptr(), n, outer, inner, 1, 1.0 / n, 0) == 0
    torch.cuda.synchronize()
    assert (torch.linalg.vector_norm(z - x) / torch.linalg.vector_norm(x)).item() <= 2e-6


def test_torch_layer_matches_torch_fft(cuda):
    import torch
    import bfly
    x = _cplx((3, 256, 512), 5, cuda)
    for norm in (None, "ortho", "forward"):
        ref2 = torch.fft.fft2(x, norm=norm)
        got2 = bfly.fft2(x, norm=norm)
        assert (torch.linalg.vector_norm(got2 - ref2) / torch.linalg.vector_norm(ref2)).item() <= 4e-6
        back = bfly.ifft2(got2, norm=norm)
        assert (torch.linalg.vector_norm(back - x) / torch.linalg.vector_norm(x)).item() <= 4e-6
        for dim in (0, 1, -2):
            if x.shape[dim] < 32:
                continue
            ref = torch.fft.fft(x, dim=dim, norm=norm)
            got = bfly.fft(x, dim=dim, norm=norm)
            assert (torch.linalg.vector_norm(got - ref) / torch.linalg.vector_norm(ref)).item() <= 3e-6
            back = bfly.ifft(got, dim=dim, norm=norm)
            assert (torch.linalg.vector_norm(back - x) / torch.linalg.vector_norm(x)).item() <= 3e-6


def test_autograd_2d_and_axis(cuda):
    """Gradients of sum(w * |X|^2) through fft2 and fft(dim=1) match torch.fft's."""
    import torch
    import bfly
    x0 = _cplx((2, 64, 128), 9, cuda)
    g = torch.Generator(device=cuda).manual_seed(10)
    w = torch.rand(2, 64, 128, device=cuda, generator=g)
    for ours, theirs in ((lambda t: bfly.fft2(t, norm="ortho"), lambda t: torch.fft.fft2(t, norm="ortho")),
                         (lambda t: bfly.fft(t, dim=1), lambda t: torch.fft.fft(t, dim=1)),
                         (lambda t: bfly.ifft2(t), lambda t: torch.fft.ifft2(t))):
        xa = x0.clone().requires_grad_(True)
        xb = x0.clone().requires_grad_(True)
        (w * ours(xa).abs() ** 2).sum().backward()
        (w * theirs(xb).abs() ** 2).sum().backward()
        rel = (torch.linalg.vector_norm(xa.grad - xb.grad) / torch.linalg.vector_norm(xb.grad)).item()
        assert rel <= 1e-5, rel


def test_unsupported_shapes_raise(cuda):
    import torch
    import bfly
    with pytest.raises(bfly.BflyError):
        bfly.fft2(_cplx((16, 64), 1, cuda))           # ny below the column envelope
    with pytest.raises(bfly.BflyError):
        bfly.fft(_cplx((8192, 4), 1, cuda), dim=0)    # strided n above 4096
    with pytest.raises(ValueError):
        bfly.fft2(torch.zeros(64, dtype=torch.complex64, device=cuda))


@pytest.mark.parametrize("ny,nx", [(32, 64), (256, 256), (1024, 128), (64, 8192), (4096, 64)])
def test_real_2d_matches_fp64(plan, cuda, ny, nx):
    """rfft2 / irfft2 layouts of numpy: [b][ny][nx] real <-> [b][ny][nx/2+1] complex."""
    import torch
    batch = 2
    g = torch.Generator(device=cuda).manual_seed(ny + nx)
    x = torch.rand(batch, ny, nx, device=cuda, generator=g) * 2 - 1
    X = torch.empty(batch, ny, nx // 2 + 1, dtype=torch.complex64, device=cuda)
    assert plan.exec_r2c_2d(x.data_ptr(), X.data_ptr(), ny, nx, batch, 1.0, 0) == 0
    torch.cuda.synchronize()
    ref = np.fft.rfft2(x.cpu().numpy().astype(np.float64))
    assert _rel_mats(X.cpu().numpy(), ref) <= 2e-6
    Xc = X.clone()
    back = torch.empty_like(x)
    assert plan.exec_c2r_2d(X.data_ptr(), back.data_ptr(), ny, nx, batch, 1.0 / (ny * nx), 0) == 0
    torch.cuda.synchronize()
    assert torch.equal(X, Xc)                       # the input half spectrum is not modified
    refb = np.fft.irfft2(ref, s=(ny, nx))
    d = np.linalg.norm((back.cpu().numpy() - refb).reshape(batch, -1), axis=-1)
    assert float((d / np.linalg.norm(refb.reshape(batch, -1), axis=-1)).max()) <= 3e-6


def test_real_2d_torch_layer_and_autograd(cuda):
    import torch
    import bfly
    g = torch.Generator(device=cuda).manual_seed(12)
    x0 = torch.randn(3, 64, 128, device=cuda, generator=g)
    for norm in (None, "ortho", "forward"):
        ref = torch.fft.rfft2(x0, norm=norm)
        got = bfly.rfft2(x0, norm=norm)
        assert (torch.linalg.vector_norm(got - ref) / torch.linalg.vector_norm(ref)).item() <= 3e-6
        back = bfly.irfft2(got, norm=norm)
        assert (torch.linalg.vector_norm(back - x0) / torch.linalg.vector_norm(x0)).item() <= 3e-6
    w = torch.rand(3, 64, 65, device=cuda, generator=g)
    xa, xb = x0.clone().requires_grad_(True), x0.clone().requires_grad_(True)
    (w * bfly.rfft2(xa, norm="ortho").abs() ** 2).sum().backward()
    (w * torch.fft.rfft2(xb, norm="ortho").abs() ** 2).sum().backward()
    assert (torch.linalg.vector_norm(xa.grad - xb.grad) / torch.linalg.vector_norm(xb.grad)).item() <= 1e-5
    X0 = torch.fft.rfft2(x0)
    wr = torch.rand(3, 64, 128, device=cuda, generator=g)
    Xa, Xb = X0.clone().requires_grad_(True), X0.clone().requires_grad_(True)
    (wr * bfly.irfft2(Xa) ** 2).sum().backward()
    (wr * torch.fft.irfft2(Xb) ** 2).sum().backward()
    assert (torch.linalg.vector_norm(Xa.grad - Xb.grad) / torch.linalg.vector_norm(Xb.grad)).item() <= 1e-5
