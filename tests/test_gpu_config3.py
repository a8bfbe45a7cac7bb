"""Mixed DCT-II / DST-I / DHT transforms at [3,256,384,320] (extra dim 3),
f32 and f64, on the 2x2 grid and the reference's 6-rank grid (2x3):

* real data through ``MixedC2cPlan`` with a zero imaginary part (the plan a
  reference caller builds: only ``MixedC2cPlan`` holds a DHT axis beside
  DCT/DST axes, distributed/mixed.rs:92-101), and through ``R2rPlan`` with a
  "Dht" axis (this library's real-valued form of the same transform);
* complex data through ``MixedC2cPlan``;
* forward, raw backward and normalised inverse, each against float64;
* the affine remap of the spectrum (sign -1 on axis 1, offsets 0 and 383),
  bit-exact.

Reference: separable float64 transforms on the host (scipy's unnormalised
FFTW-convention DCT-II / DST-I and the DHT as Re F - Im F), computed once
per module.  Bound: rel-L2 <= 1e-6 log2 N (f32) / 1e-14 log2 N (f64),
N = 256*384*320.  Each case prints the errors it measured.
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
# product of the raw backward's normalisation factors: DCT-II 2n, DST-I 2(n+1), DHT n
RAW_SCALE = (2 * 256) * (2 * (384 + 1)) * 320


def reference(x):
    """float64 separable DCT-II (axis 0), DST-I (axis 1), DHT (axis 2); batch axis first."""
    y = sf.dct(x, type=2, axis=1, workers=-1)
    y = sf.dst(y, type=1, axis=2, workers=-1)
    f = sf.fft(y, axis=3, workers=-1)
    return f.real - f.imag


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


_CACHE = {}


def fields():
    """Seed-2 N(0,1) data: the real field is the real part of the complex one
    (both drawn from a fresh default_rng(2)), with their float64 transforms."""
    if not _CACHE:
        rng = np.random.default_rng(2)
        re = rng.standard_normal(EXTRA + SHAPE)
        im = rng.standard_normal(EXTRA + SHAPE)
        _CACHE.update(re=re, im=im, ref_re=reference(re), ref_im=reference(im))
    return _CACHE


def make_plan(form, dims, real_dtype):
    topo = pb.MpiTopology(dims)
    cdt = torch.complex64 if real_dtype == torch.float32 else torch.complex128
    if form == "r2r":
        return pb.R2rPlan.from_shape(topo, SHAPE, EXTRA, KINDS, dtype=real_dtype)
    return pb.MixedC2cPlan.from_shape(topo, SHAPE, EXTRA, KINDS, dtype=cdt)


@pytest.mark.parametrize("dims", [(2, 2), (2, 3)])
@pytest.mark.parametrize("real_dtype", [torch.float32, torch.float64], ids=["f32", "f64"])
@pytest.mark.parametrize("form", ["mixed_real", "mixed_complex", "r2r"])
def test_config3_mixed_kinds_full_size(form, real_dtype, dims):
    f = fields()
    plan = make_plan(form, dims, real_dtype)
    npr = np.float32 if real_dtype == torch.float32 else np.float64
    if form == "r2r":
        x = f["re"].astype(npr)
        ref = f["ref_re"]
        xd = x.astype(np.float64)
    elif form == "mixed_real":
        x = f["re"].astype(npr).astype(np.complex64 if npr == np.float32 else np.complex128)
        ref = f["ref_re"]
        xd = x.real.astype(np.float64)
    else:
        x = (f["re"] + 1j * f["im"]).astype(np.complex64 if npr == np.float32 else np.complex128)
        ref = f["ref_re"] + 1j * f["ref_im"]
        xd = x.astype(np.complex128)
    # in f32 the reference is that of the unrounded float64 field: rounding the
    # input to f32 changes the transform by about 6e-8 relative, far inside the bound
    src = plan.input_pencil.scatter(torch.from_numpy(x).cuda(), 3).contiguous()
    out = plan.allocate_output()
    plan.forward(src, out)
    got = plan.output_pencil.gather(out, 3).cpu().numpy()
    lg = math.log2(np.prod(SHAPE))
    bound = (1e-6 if npr == np.float32 else 1e-14) * lg
    err_fwd = rel(got, ref)
    back = plan.allocate_input()
    plan.backward(out, back)
    err_bwd = rel(plan.input_pencil.gather(back, 3).cpu().numpy() / RAW_SCALE, xd)
    plan.inverse(out, back)
    err_inv = rel(plan.input_pencil.gather(back, 3).cpu().numpy(), xd)
    print(f"\nconfig 3 {form} {'f32' if npr == np.float32 else 'f64'} grid {dims[0]}x{dims[1]}: forward "
          f"{err_fwd:.3e}, raw backward/S {err_bwd:.3e}, inverse {err_inv:.3e}, bound {bound:.2e}")
    assert err_fwd <= bound
    assert err_bwd <= bound
    assert err_inv <= bound
    if form == "r2r":
        return
    # affine remap of the spectrum: k -> -k and the mirror k -> 383 - k on axis 1, bit-exact
    glob = plan.output_pencil.gather(out, 3)
    dst_pencil = pb.Pencil(pb.MpiTopology(dims), SHAPE, (0, 1))
    for offsets in ((0, 0, 0), (0, 383, 0)):
        remap = pb.SpatialRemapPlan.prepare(plan.output_pencil, dst_pencil, 3, (1, -1, 1), offsets, out.dtype)
        moved = torch.empty(dst_pencil.total(3), dtype=out.dtype, device="cuda")
        remap.apply(out, moved)
        idx = (offsets[1] - torch.arange(384, device="cuda")) % 384
        assert torch.equal(dst_pencil.gather(moved, 3), glob[:, :, idx, :])
