"""The headline plan exactly as benchmarked: R2C f32 [512,512,512] on the 4x8
virtual grid (reduction on the last axis -> 257), field A = uniform(-1,1)
from numpy ``default_rng(1)``.

* forward spectrum against torch's float64 ``rfftn`` of the same field;
* normalised inverse of the library's own spectrum against float64 ``irfftn``
  of that spectrum, and the round trip against the field;
* field B (16 random-phase cosines, ``default_rng(1)`` continued) against its
  known 32-bin spectrum.

Bound: rel-L2 <= 1e-6 * log2(N) = 2.7e-5.  The float64 FFTs are the checker
only (torch on the same GPU).  Each test prints the error it measured.
"""

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

import pencil_b200 as pb  # noqa: E402

SHAPE = (512, 512, 512)
GRID = (4, 8)
BOUND = 1e-6 * math.log2(512 ** 3)


def rel(a, b):
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


@pytest.fixture(scope="module")
def headline():
    plan = pb.R2cPlan.from_shape(pb.MpiTopology(GRID), SHAPE, (), dtype=torch.float32)
    assert plan.step_kernels(0) == ["pow2", "pow2", "pow2"]
    rng = np.random.default_rng(1)
    xa = torch.from_numpy(rng.uniform(-1.0, 1.0, SHAPE).astype(np.float32)).cuda()
    yield plan, xa
    plan.close()


def test_config2_forward_and_inverse_against_float64(headline):
    plan, xa = headline
    ws = plan.allocate_workspace()
    src = plan.input_pencil.scatter(xa).contiguous()
    spec = plan.allocate_output()
    plan.forward(src, spec, ws)
    got = plan.output_pencil.gather(spec)[0]
    ref = torch.fft.rfftn(xa.double())
    err_fwd = rel(got.to(torch.complex128), ref)
    del ref
    back = plan.allocate_input()
    plan.inverse(spec, back, ws)
    back_g = plan.input_pencil.gather(back)[0].double()
    ref_inv = torch.fft.irfftn(got.to(torch.complex128), s=SHAPE)
    err_inv = rel(back_g, ref_inv)
    err_rt = rel(back_g, xa.double())
    print(f"\nconfig 2 (512^3 R2C f32, 4x8): forward rel-L2 {err_fwd:.3e}, inverse rel-L2 {err_inv:.3e}, "
          f"round trip {err_rt:.3e}, bound {BOUND:.2e}")
    assert err_fwd <= BOUND
    assert err_inv <= BOUND
    assert err_rt <= BOUND


def test_config2_field_b_known_spectrum(headline):
    plan, _ = headline
    # field B continues the generator after field A (as the benchmark draws it)
    rng = np.random.default_rng(1)
    rng.uniform(-1.0, 1.0, SHAPE)
    kvec = rng.integers(0, SHAPE[0] // 2, size=(16, 3))
    phase = rng.uniform(0.0, 2 * math.pi, 16)
    axes = [torch.arange(n, device="cuda", dtype=torch.float64) for n in SHAPE]
    fb = torch.zeros(SHAPE, dtype=torch.float64, device="cuda")
    for m in range(16):
        th = (2 * math.pi * int(kvec[m, 0]) / SHAPE[0] * axes[0])[:, None, None] + \
             (2 * math.pi * int(kvec[m, 1]) / SHAPE[1] * axes[1])[None, :, None] + \
             (2 * math.pi * int(kvec[m, 2]) / SHAPE[2] * axes[2])[None, None, :]
        fb += torch.cos(th + float(phase[m]))
    src = plan.input_pencil.scatter(fb.float()).contiguous()
    del fb
    spec = plan.allocate_output()
    plan.forward(src, spec)
    got = plan.output_pencil.gather(spec)[0].to(torch.complex128)
    exp = torch.zeros_like(got)
    ntot = float(np.prod(SHAPE))
    for m in range(16):
        k = [int(v) for v in kvec[m]]
        pk = tuple(v % n for v, n in zip(k, SHAPE))
        mk = tuple((-v) % n for v, n in zip(k, SHAPE))
        for idx, sgn in ((pk, 1.0), (mk, -1.0)):
            if idx[2] <= SHAPE[2] // 2:
                exp[idx] += (ntot / 2) * complex(math.cos(phase[m]), sgn * math.sin(phase[m]))
    err = rel(got, exp)
    print(f"\nconfig 2 field B: known-spectrum rel-L2 {err:.3e}, bound {BOUND:.2e}")
    assert err <= BOUND
