"""ADI heat diffusion (GPU): forward steps against the oracle's ADI step
(oracle_adi_f64, pinned on the CPU to the reference's adi_orig.c), CUDA-graph
replay against eager steps, and the checkpointed adjoint against autograd
through a dense torch restatement of the step."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from tridsolver_b200.adi import ADI, COEFFS  # noqa: E402
from oracle import oracle  # noqa: E402

from helpers import rel_err  # noqa: E402


def ref_init(nz, ny, nx):
    u = np.zeros((nz, ny, nx))
    u[[0, -1], :, :] = 1
    u[:, [0, -1], :] = 1
    u[:, :, [0, -1]] = 1
    return u


@pytest.mark.parametrize("kind", ["plain", "reference"])
def test_adi_64cube_10_steps(kind):
    nz = ny = nx = 64
    lam = 1.0
    if kind == "reference":
        u0 = ref_init(nz, ny, nx)
    else:
        u0 = np.random.default_rng(1).uniform(0, 1, (nz, ny, nx))
    a, b, c = COEFFS[kind][0](lam)
    expect = oracle.adi(u0.ravel(), nx, ny, nz, 10, lam, a, b, c).reshape(nz, ny, nx)
    u = torch.from_numpy(u0.copy()).cuda()
    ADI((nz, ny, nx), lam, kind).step(u, 10)
    assert rel_err(u.cpu().numpy(), expect) <= 1e-12


@pytest.mark.parametrize("shape", [(30, 17, 45), (5, 3, 2), (128, 1, 7)])
def test_adi_odd_shapes(shape):
    nz, ny, nx = shape
    u0 = np.random.default_rng(2).uniform(0, 1, shape)
    a, b, c = COEFFS["plain"][0](0.7)
    expect = oracle.adi(u0.ravel(), nx, ny, nz, 3, 0.7, a, b, c).reshape(shape)
    u = torch.from_numpy(u0.copy()).cuda()
    ADI(shape, 0.7).step(u, 3)
    assert rel_err(u.cpu().numpy(), expect) <= 1e-12


def test_adi_graph_replay_matches_eager():
    shape = (128, 128, 128)
    u0 = torch.rand(shape, dtype=torch.float64, device="cuda", generator=torch.Generator(
        device="cuda").manual_seed(3))
    u1, u2 = u0.clone(), u0.clone()
    ADI(shape, 1.0).step(u1, 12)
    ADI(shape, 1.0).run(u2, 12, graph=True)
    torch.cuda.synchronize()
    assert torch.equal(u1, u2)


# ------------------------------------------------------------- adjoint --
def _dense_solve_axis(v, axis, lam, kind, mask):
    ca, cb, cc = COEFFS[kind][0](lam)
    vm = v.movedim(axis, -1)
    mm = mask.movedim(axis, -1)
    n = vm.shape[-1]
    lines = vm.reshape(-1, n)
    ml = mm.reshape(-1, n)
    one = torch.ones_like(lines)
    zero = torch.zeros_like(lines)
    av = torch.where(ml, ca * one, zero)
    bv = torch.where(ml, cb * one, one)
    cv = torch.where(ml, cc * one, zero)
    A = torch.diag_embed(bv) + torch.diag_embed(av[:, 1:], -1) + torch.diag_embed(cv[:, :-1], 1)
    x = torch.linalg.solve(A, lines.unsqueeze(-1)).squeeze(-1)
    return x.reshape(vm.shape).movedim(-1, axis)


def _dense_step(u, lam, kind, mask):
    r = torch.zeros_like(u)
    r[1:-1, 1:-1, 1:-1] = lam * (u[2:, 1:-1, 1:-1] + u[:-2, 1:-1, 1:-1] + u[1:-1, 2:, 1:-1] +
                                 u[1:-1, :-2, 1:-1] + u[1:-1, 1:-1, 2:] + u[1:-1, 1:-1, :-2] -
                                 6.0 * u[1:-1, 1:-1, 1:-1])
    du1 = _dense_solve_axis(r, 2, lam, kind, mask)
    du2 = _dense_solve_axis(du1, 1, lam, kind, mask)
    du3 = _dense_solve_axis(du2, 0, lam, kind, mask)
    return u + du3


@pytest.mark.parametrize("kind", ["plain", "reference"])
def test_adi_checkpointed_adjoint_against_dense_autograd(kind):
    shape = (7, 9, 10)
    steps, every, lam = 6, 4, 0.8
    g = torch.Generator(device="cuda").manual_seed(4)
    u0 = torch.rand(shape, dtype=torch.float64, device="cuda", generator=g)
    loss, du0, dlam = ADI(shape, lam, kind).grad_final_norm(u0, steps, every)

    mask = torch.zeros(shape, dtype=torch.bool, device="cuda")
    mask[1:-1, 1:-1, 1:-1] = True
    ur = u0.clone().requires_grad_(True)
    lr = torch.tensor(lam, dtype=torch.float64, device="cuda", requires_grad=True)
    u = ur
    for _ in range(steps):
        u = _dense_step(u, lr, kind, mask)
    lref = torch.linalg.vector_norm(u)
    lref.backward()
    assert abs(float(loss) - float(lref.detach())) <= 1e-12 * abs(float(lref.detach()))
    assert rel_err(du0.cpu().numpy(), ur.grad.cpu().numpy()) <= 1e-10
    assert abs(float(dlam) - float(lr.grad)) <= 1e-10 * max(1.0, abs(float(lr.grad)))


def test_adi_lambda_gradient_finite_difference():
    shape = (16, 16, 16)
    steps, every, lam, h = 8, 3, 1.0, 1e-6
    u0 = torch.rand(shape, dtype=torch.float64, device="cuda",
                    generator=torch.Generator(device="cuda").manual_seed(5))
    _, _, dlam = ADI(shape, lam).grad_final_norm(u0, steps, every)

    def final_norm(l):
        u = u0.clone()
        ADI(shape, l).step(u, steps)
        return float(torch.linalg.vector_norm(u))

    fd = (final_norm(lam + h) - final_norm(lam - h)) / (2 * h)
    assert abs(fd - float(dlam)) <= 1e-7 * max(1.0, abs(fd))
