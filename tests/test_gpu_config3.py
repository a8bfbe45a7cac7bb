"""Mixed DCT-II / DST-I / DHT transforms at [3,256,384,320] (extra dim 3) on
the reference's 6-rank grid (2x3), real f32 and complex f32, and the affine
remap of the result (sign -1 on axis 1, offsets 0 and 383), bit-exact.

Full-size reference: separable float64 transforms on the host (scipy's
unnormalised FFTW-convention DCT-II / DST-I and the DHT as Re F - Im F).
"""

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

import scipy.fft as sf  # noqa: E402

import pencil_b200 as pb  # noqa: E402

SHAPE = (256, 384, 320)
EXTRA = (3,)
KINDS = ("DctII", "DstI", "Dht")


def reference(x):
    """float64 separable DCT-II (axis 0), DST-I (axis 1), DHT (axis 2); batch axis first."""
    y = sf.dct(x, type=2, axis=1, workers=-1)
    y = sf.dst(y, type=1, axis=2, workers=-1)
    f = sf.fft(y, axis=3, workers=-1)
    return f.real - f.imag


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


@pytest.mark.parametrize("cplx", [False, True])
def test_config3_mixed_kinds_full_size(cplx):
    rng = np.random.default_rng(2)
    topo = pb.MpiTopology((2, 3))
    if cplx:
        plan = pb.MixedC2cPlan.from_shape(topo, SHAPE, EXTRA, KINDS, dtype=torch.complex64)
        x = (rng.standard_normal(EXTRA + SHAPE) + 1j * rng.standard_normal(EXTRA + SHAPE)).astype(np.complex64)
        xt = torch.from_numpy(x).cuda()
    else:
        plan = pb.R2rPlan.from_shape(topo, SHAPE, EXTRA, KINDS, dtype=torch.float32)
        x = rng.standard_normal(EXTRA + SHAPE).astype(np.float32)
        xt = torch.from_numpy(x).cuda()
    src = plan.input_pencil.scatter(xt, 3).contiguous()
    out = plan.allocate_output()
    plan.forward(src, out)
    got = plan.output_pencil.gather(out, 3).cpu().numpy()
    xd = x.astype(np.complex128 if cplx else np.float64)
    ref = reference(xd.real) + (1j * reference(xd.imag) if cplx else 0)
    bound = 1e-6 * math.log2(np.prod(SHAPE))
    assert rel(got, ref) <= bound
    # raw backward of the forward scales by the product of normalisation factors
    back = plan.allocate_input()
    plan.backward(out, back)
    s = (2 * 256) * (2 * (384 + 1)) * 320
    assert rel(plan.input_pencil.gather(back, 3).cpu().numpy() / s, xd) <= bound
    plan.inverse(out, back)
    assert rel(plan.input_pencil.gather(back, 3).cpu().numpy(), xd) <= bound
    # affine remap of the spectrum: k -> -k and the mirror k -> 383 - k on axis 1, bit-exact
    dtype = out.dtype
    glob = plan.output_pencil.gather(out, 3)
    dst_pencil = pb.Pencil(topo, SHAPE, (0, 1))
    for offsets in ((0, 0, 0), (0, 383, 0)):
        remap = pb.SpatialRemapPlan.prepare(plan.output_pencil, dst_pencil, 3, (1, -1, 1), offsets, dtype)
        moved = torch.empty(dst_pencil.total(3), dtype=dtype, device="cuda")
        remap.apply(out, moved)
        idx = (offsets[1] - torch.arange(384, device="cuda")) % 384
        assert torch.equal(dst_pencil.gather(moved, 3), glob[:, :, idx, :])
