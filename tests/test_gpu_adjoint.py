"""Adjoint gradients of a Jacobi-PCG solve (celg_pcg_adjoint and
celg_diffusion7_face_grad), wrapped in a torch.autograd.Function that lives
only here in the test harness.

Loss L = 0.5 ||x(g, b) - x_target||^2 with x from A(k) x = b, k = exp(g) per
face of a 7-point diffusion operator.  Checked three ways: bit-exact against
the oracle's adjoint (tree order), against central finite differences along
random unit directions, and through torch autograd."""
import numpy as np
import pytest

from cel_v3_b200 import synth
from oracle import celref as R

pytestmark = pytest.mark.gpu

GRID = (10, 11, 12)
EPS = 1e-13


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def split(g, grid):
    nx, ny, nz = grid
    cx, cy, cz = synth.face_counts(nx, ny, nz)
    return g[:cx], g[cx:cx + cy], g[cx + cy:]


def solve(celgpu, h, torch, g, b):
    """x(g, b) on the GPU; returns (matrix, x)."""
    kx, ky, kz = split(np.exp(g), GRID)
    rp, ci, v = synth.diffusion7(*GRID, kx, ky, kz)
    m = h.matrix_from_csr(rp, ci, v).jacobi()
    x = dev(torch, np.zeros(b.size))
    info = h.pcg_jacobi(m, dev(torch, b).data_ptr(), x.data_ptr(), eps_rel=EPS, iter_max=5000)
    assert info.status == celgpu.OK
    return m, (rp, ci, v), x


def loss_and_grads(celgpu, h, torch, g, b, xt):
    m, (rp, ci, v), x = solve(celgpu, h, torch, g, b)
    gx = x - dev(torch, xt)
    lam = torch.zeros_like(x)
    gA = torch.zeros(int(rp[-1]), dtype=torch.float64, device="cuda")
    h.pcg_adjoint(m, x.data_ptr(), gx.data_ptr(), lam.data_ptr(), gA.data_ptr(), eps_rel=EPS,
                  iter_max=5000)
    cx, cy, cz = synth.face_counts(*GRID)
    gk = torch.zeros(cx + cy + cz, dtype=torch.float64, device="cuda")
    h.diffusion7_face_grad(*GRID, lam.data_ptr(), x.data_ptr(), gk.data_ptr(),
                           gk[cx:].data_ptr(), gk[cx + cy:].data_ptr())
    L = 0.5 * float((gx * gx).sum())
    m.destroy()
    return L, x.cpu().numpy(), lam.cpu().numpy(), gA.cpu().numpy(), gk.cpu().numpy(), (rp, ci, v)


@pytest.fixture(scope="module")
def problem():
    rng = np.random.default_rng(6)
    nx, ny, nz = GRID
    cx, cy, cz = synth.face_counts(nx, ny, nz)
    g = rng.standard_normal(cx + cy + cz)
    r7 = np.random.default_rng(7)
    b = r7.uniform(-1.0, 1.0, nx * ny * nz)
    xt = r7.random(nx * ny * nz)
    return g, b, xt


def test_adjoint_bitexact_against_oracle(gpu, problem):
    celgpu, h, torch = gpu
    g, b, xt = problem
    L, x, lam, gA, gk, (rp, ci, v) = loss_and_grads(celgpu, h, torch, g, b, xt)
    A = R.Matrix(rp, ci, v)
    J = R.jacobi(R.diag(rp, ci, v))
    lam_o, _ = R.pcg_jacobi(A, J, x - xt, eps_rel=EPS, iter_max=5000, red=R.RED_TREE)
    assert np.array_equal(lam, lam_o)
    rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))
    assert np.array_equal(gA, -(lam[rows] * x[ci]))
    # face gradients from the pattern gradient (contraction with dA/dk_f)
    nx, ny, nz = GRID
    cell = lambda X, Y, Z: X + nx * (Y + ny * Z)
    gx_, gy_, gz_ = split(gk, GRID)
    Xc, Yc, Zc = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    # an interior x-face between (X, Y, Z) and (X+1, Y, Z)
    for (X, Y, Z) in [(0, 0, 0), (3, 4, 5), (nx - 2, ny - 1, nz - 1)]:
        i, j = cell(X, Y, Z), cell(X + 1, Y, Z)
        f = (X + 1) + (nx + 1) * (Y + ny * Z)
        assert gx_[f] == -((lam[i] - lam[j]) * (x[i] - x[j]))
    # a boundary z-face of cell (2, 3, nz-1)
    i = cell(2, 3, nz - 1)
    assert gz_[2 + nx * (3 + ny * nz)] == -(lam[i] * x[i])


def test_adjoint_matches_central_differences(gpu, problem):
    celgpu, h, torch = gpu
    g, b, xt = problem
    L, x, lam, gA, gk, _ = loss_and_grads(celgpu, h, torch, g, b, xt)
    dLdg = np.exp(g) * gk
    rng = np.random.default_rng(64)
    step = 1e-6
    for _ in range(8):
        d = rng.standard_normal(g.size)
        d /= np.linalg.norm(d)
        Lp = loss_and_grads(celgpu, h, torch, g + step * d, b, xt)[0]
        Lm = loss_and_grads(celgpu, h, torch, g - step * d, b, xt)[0]
        fd = (Lp - Lm) / (2 * step)
        assert abs(fd - dLdg @ d) <= 1e-5 * max(abs(fd), np.abs(dLdg).max())
    # dL/db along a direction
    e = rng.standard_normal(b.size)
    e /= np.linalg.norm(e)
    Lp = loss_and_grads(celgpu, h, torch, g, b + step * e, xt)[0]
    Lm = loss_and_grads(celgpu, h, torch, g, b - step * e, xt)[0]
    assert abs((Lp - Lm) / (2 * step) - lam @ e) <= 1e-5 * np.abs(lam).max()


def test_torch_autograd_wrapper(gpu, problem):
    celgpu, h, torch = gpu
    g, b, xt = problem

    class PCGSolve(torch.autograd.Function):
        """x = A(exp(g))^{-1} b; backward through celg_pcg_adjoint."""

        @staticmethod
        def forward(ctx, gt, bt):
            m, _, x = solve(celgpu, h, torch, gt.detach().cpu().numpy(), bt.detach().cpu().numpy())
            ctx.save_for_backward(gt, x)
            ctx.m = m
            return x.clone()

        @staticmethod
        def backward(ctx, gx):
            gt, x = ctx.saved_tensors
            gx = gx.contiguous()
            lam = torch.zeros_like(x)
            h.pcg_adjoint(ctx.m, x.data_ptr(), gx.data_ptr(), lam.data_ptr(), eps_rel=EPS,
                          iter_max=5000)
            gk = torch.zeros_like(gt)
            cx, cy, cz = synth.face_counts(*GRID)
            h.diffusion7_face_grad(*GRID, lam.data_ptr(), x.data_ptr(), gk.data_ptr(),
                                   gk[cx:].data_ptr(), gk[cx + cy:].data_ptr())
            ctx.m.destroy()
            return torch.exp(gt) * gk, lam

    gt = torch.tensor(g, device="cuda", requires_grad=True)
    bt = torch.tensor(b, device="cuda", requires_grad=True)
    x = PCGSolve.apply(gt, bt)
    loss = 0.5 * ((x - torch.tensor(xt, device="cuda")) ** 2).sum()
    loss.backward()
    L, _, lam, _, gk, _ = loss_and_grads(celgpu, h, torch, g, b, xt)
    assert np.array_equal(bt.grad.cpu().numpy(), lam)
    # exp is evaluated by torch on the GPU here and by numpy above: equal to an ulp
    assert np.allclose(gt.grad.cpu().numpy(), np.exp(g) * gk, rtol=1e-14, atol=0)
