"""Long columns (1024, 2048, 4096 points) through the column kernel, against FP64 numpy.

The column kernel transforms strips of C consecutive columns per CTA (16 / 8 / 4 columns at
these lengths), so the shapes below cover partial last strips (ncols not a multiple of C), rows
narrower than a strip, many strips per launch and in-place calls.  Tolerance: rel L2 <= 1e-6
per column (the single-pass gate) and <= 2e-6 for 2-D transforms."""
import numpy as np
import pytest

import oracle.fft_oracle as O

pytestmark = pytest.mark.gpu


def _cplx(shape, seed, cuda):
    import torch
    g = torch.Generator(device=cuda).manual_seed(seed)
    return torch.randn(*shape, dtype=torch.complex64, device=cuda, generator=g)


@pytest.mark.parametrize("n", [1024, 2048, 4096])
@pytest.mark.parametrize("outer,inner", [(1, 2), (3, 130), (2, 1024), (40, 64)])
@pytest.mark.parametrize("direction", [-1, 1])
def test_long_columns_match_fp64(plan, cuda, n, outer, inner, direction):
    import torch
    x = _cplx((outer, n, inner), 5 * n + inner + outer, cuda)
    y = torch.full_like(x, float("nan"))
    scale = 1.0 if direction < 0 else 1.0 / n
    assert plan.exec_c2c_axis(x.data_ptr(), y.data_ptr(), n, outer, inner, direction, scale, 0) == 0
    torch.cuda.synchronize()
    xd = x.cpu().numpy().astype(np.complex128)
    ref = np.fft.fft(xd, axis=1) if direction < 0 else np.fft.ifft(xd, axis=1)
    got = np.moveaxis(y.cpu().numpy(), 1, -1).reshape(-1, n)
    assert np.isfinite(got).all()
    assert O.rel_l2_rows(got, np.moveaxis(ref, 1, -1).reshape(-1, n)) <= 1e-6


@pytest.mark.parametrize("ny,nx,batch", [(1024, 1024, 2), (2048, 512, 3), (4096, 256, 2), (1024, 96, 5)])
def test_long_column_2d_and_in_place(plan, cuda, ny, nx, batch):
    import torch
    x = _cplx((batch, ny, nx), ny + nx, cuda)
    y = torch.empty_like(x)
    assert plan.exec_c2c_2d(x.data_ptr(), y.data_ptr(), ny, nx, batch, -1, 1.0, 0) == 0
    z = x.clone()
    assert plan.exec_c2c_2d(z.data_ptr(), z.data_ptr(), ny, nx, batch, -1, 1.0, 0) == 0
    torch.cuda.synchronize()
    assert torch.equal(y, z)
    ref = np.fft.fft2(x.cpu().numpy().astype(np.complex128))
    d = np.linalg.norm((y.cpu().numpy() - ref).reshape(batch, -1), axis=-1)
    assert float((d / np.linalg.norm(ref.reshape(batch, -1), axis=-1)).max()) <= 2e-6
    assert plan.exec_c2c_2d(y.data_ptr(), z.data_ptr(), ny, nx, batch, 1, 1.0 / (ny * nx), 0) == 0
    torch.cuda.synchronize()
    assert (torch.linalg.vector_norm(z - x) / torch.linalg.vector_norm(x)).item() <= 4e-6
