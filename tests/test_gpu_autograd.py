"""Differentiation through the library (adjoint kernels behind torch.autograd).

* f64 central finite differences (h = 1e-6, 32 random directions) of
  L(u) = sum |k|^2 |R2C(u)|^2 and of a spectral Poisson solve followed by C2R;
* the VJP against the oracle's restatement of the reference's raw
  ``backward`` (C2C: the adjoint is the raw opposite-sign transform; R2C: raw
  C2R of the cotangent with interior bins halved);
* at full size, R2C f32 [384,384,384] on a 4x8 grid, the gradient of the loss
  and the Poisson solve against torch's float64 FFT autograd (checker only).
"""

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

import pencil_b200 as pb  # noqa: E402
from pencil_b200 import autograd as pba  # noqa: E402


def k2_loss(plan, u):
    spec = pba.forward(plan, u)
    weighted = pba.spectral_multiply(plan, spec, "k2")
    return torch.sum((spec.conj() * weighted).real)


def poisson_loss(plan, u, w):
    phi = pba.inverse(plan, pba.spectral_multiply(plan, pba.forward(plan, u), "poisson"))
    return torch.sum(w * phi * phi)


@pytest.mark.parametrize("shape,dims", [((12, 10, 8), (2, 2)), ((9, 8, 16), (3, 2)), ((16, 32, 64), (2, 4))])
def test_vjp_matches_f64_central_differences(shape, dims):
    torch.manual_seed(3)
    plan = pb.R2cPlan.from_shape(pb.MpiTopology(dims), shape, (), dtype=torch.float64)
    n = plan.info.input_elems
    u = torch.randn(n, dtype=torch.float64, device="cuda", requires_grad=True)
    w = torch.rand(n, dtype=torch.float64, device="cuda")
    h = 1e-6
    for loss in (lambda x: k2_loss(plan, x), lambda x: poisson_loss(plan, x, w)):
        val = loss(u)
        (grad,) = torch.autograd.grad(val, u)
        worst = 0.0
        with torch.no_grad():
            for _ in range(32):
                v = torch.randn(n, dtype=torch.float64, device="cuda")
                fd = (loss(u + h * v) - loss(u - h * v)) / (2 * h)
                an = torch.dot(grad, v)
                # directional error relative to the Cauchy-Schwarz scale |grad||v|
                scale = float(torch.linalg.vector_norm(grad) * torch.linalg.vector_norm(v))
                worst = max(worst, float(abs(fd - an)) / scale)
        assert worst <= 1e-8, worst


def test_vjp_matches_the_reference_backward():
    """The VJP kernels against the oracle's restatement of the reference's raw
    ``backward`` (execute_inverse with backward locals and no normalisation,
    distributed.rs:1448-1500, distributed/r2c.rs:3410-3511): for C2C the
    adjoint of forward is the raw opposite-sign transform; for R2C it is the
    raw C2R of the cotangent with the interior bins of the reduced axis
    halved."""
    import pencil_oracle as po
    from pb_testutil import oracle_pencil

    torch.manual_seed(4)
    dims, shape = (2, 2), (12, 10, 8)
    topo = pb.MpiTopology(dims)
    c2c = pb.C2cPlan.from_shape(topo, shape, (), dtype=torch.complex128)
    g = torch.randn(c2c.info.output_elems, dtype=torch.complex128, device="cuda")
    a = c2c.allocate_input()
    c2c.vjp_forward(g, a)
    route = po.c2c_route(po.Topology(dims), shape)
    locs = po.split_flat(oracle_pencil(c2c.output_pencil), g.cpu().numpy(), 1)
    exp = torch.from_numpy(po.flat_concat(po.execute_reverse(route, locs, False))).cuda()
    torch.cuda.synchronize()
    assert torch.allclose(a, exp, rtol=0, atol=1e-12 * float(exp.abs().max()))
    r2c = pb.R2cPlan.from_shape(topo, shape, (), dtype=torch.float64)
    # a cotangent the raw backward accepts: the spectrum of a real field, whose
    # DC and Nyquist planes are Hermitian in the transverse axes
    spec = r2c.allocate_output()
    r2c.forward(torch.randn(r2c.info.input_elems, dtype=torch.float64, device="cuda"), spec)
    gs = r2c.output_pencil.gather(spec)
    half = gs.clone()
    half[..., 1:4] *= 0.5  # interior bins of the reduced axis (n = 8)
    x1 = r2c.allocate_input()
    r2c.vjp_forward(r2c.output_pencil.scatter(gs).contiguous(), x1)
    route = po.r2c_route(po.Topology(dims), shape)
    hflat = r2c.output_pencil.scatter(half).contiguous().cpu().numpy()
    locs = po.split_flat(oracle_pencil(r2c.output_pencil), hflat, 1)
    exp = torch.from_numpy(po.flat_concat(po.execute_reverse(route, locs, False)).real.copy()).cuda()
    torch.cuda.synchronize()
    assert torch.allclose(x1, exp, rtol=0, atol=1e-12 * float(exp.abs().max()))


def test_full_size_384_gradient_and_poisson_against_float64():
    shape = (384, 384, 384)
    plan = pb.R2cPlan.from_shape(pb.MpiTopology((4, 8)), shape, (), dtype=torch.float32)
    gen = torch.Generator(device="cuda").manual_seed(3)
    u_glob = torch.randn(shape, generator=gen, device="cuda", dtype=torch.float32)
    u = plan.input_pencil.scatter(u_glob).contiguous().requires_grad_(True)
    loss = k2_loss(plan, u)
    (grad,) = torch.autograd.grad(loss, u)
    grad_glob = plan.input_pencil.gather(grad)[0].double()
    del grad
    # float64 reference through torch's FFT autograd (checker only)
    ud = u_glob.double().requires_grad_(True)
    spec = torch.fft.rfftn(ud)
    k = [torch.fft.fftfreq(n, d=1.0 / n, device="cuda", dtype=torch.float64) for n in shape[:2]]
    k.append(torch.arange(shape[2] // 2 + 1, device="cuda", dtype=torch.float64))
    k2 = k[0][:, None, None] ** 2 + k[1][None, :, None] ** 2 + k[2][None, None, :] ** 2
    ref_loss = torch.sum(k2 * (spec.real ** 2 + spec.imag ** 2))
    (ref_grad,) = torch.autograd.grad(ref_loss, ud)
    bound = 1e-6 * math.log2(np.prod(shape))
    assert abs(float(loss) - float(ref_loss)) / float(ref_loss) <= bound
    assert float(torch.linalg.vector_norm(grad_glob - ref_grad) / torch.linalg.vector_norm(ref_grad)) <= bound
    del ud, spec, ref_grad, grad_glob
    # spectral Poisson solve: phi = C2R(-U/|k|^2), U(0) = 0
    with torch.no_grad():
        phi = pba.inverse(plan, pba.spectral_multiply(plan, pba.forward(plan, u.detach()), "poisson"))
        phi_glob = plan.input_pencil.gather(phi)[0].double()
        uh = torch.fft.rfftn(u_glob.double())
        mult = torch.where(k2 == 0, torch.zeros_like(k2), -1.0 / torch.where(k2 == 0, torch.ones_like(k2), k2))
        ref_phi = torch.fft.irfftn(uh * mult, s=shape)
        assert float(torch.linalg.vector_norm(phi_glob - ref_phi) / torch.linalg.vector_norm(ref_phi)) <= bound
