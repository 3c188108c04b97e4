"""Adjoint form (variable kappa): the device VJP against the oracle, the
autograd rule against exact directional derivatives, and the adjoint-CG
gradient of J(kappa) = 0.5||u(kappa) - u_obs||^2 against central finite
differences (step 1e-6) and the oracle's sparse-direct adjoint gradient."""
import numpy as np
import pytest

from oracle import sumfac_oracle as O

pytestmark = pytest.mark.gpu


def setup(sf, p, deg, n, perturb=0.0, seed=0):
    model = sf.CartesianDiscreteModel((0, 1, 0, 1, 0, 1), (n, n, n), perturb=perturb, seed=seed)
    V = sf.FESpace(model, p)
    m = sf.SumFactorizationMap(3, (p,) * 3, (deg,) * 3)
    A = sf.LazyMatrix(m, V, V, sf.Measure(model, deg))
    om = O.make_map(3, p, deg)
    mesh = O.cartesian_mesh(3, n, p, om, perturb=perturb, seed=seed)
    return A, V, om, mesh


def kappa_field(seed, nc, nq):
    return np.exp(np.random.default_rng(seed).normal(0.0, 0.5, (nc, nq)))


@pytest.mark.parametrize("p,deg,n,pert", [(3, 6, 4, 0.0), (2, 4, 3, 0.2), (4, 8, 2, 0.0)])
def test_kappa_vjp_matches_oracle(sf, p, deg, n, pert):
    import torch
    A, V, om, mesh = setup(sf, p, deg, n, pert, 3)
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, mesh.n_free)
    yb = rng.uniform(-1, 1, mesh.n_free)
    kb_ref = O.kappa_vjp(om, mesh, x, yb)
    kb = A.kappa_vjp(torch.from_numpy(x).cuda(), torch.from_numpy(yb).cuda()).cpu().numpy()
    assert np.abs(kb - kb_ref).max() < 1e-12 * np.abs(kb_ref).max()
    kb32 = A.kappa_vjp(torch.from_numpy(x).cuda().float(),
                       torch.from_numpy(yb).cuda().float()).cpu().numpy()
    assert np.abs(kb32 - kb_ref).max() < 1e-4 * np.abs(kb_ref).max()


def test_autograd_rule(sf):
    """The backward pass of y = A(kappa) x equals the exact directional
    derivatives (y is linear in x and in kappa)."""
    import torch
    from ncihackaton2023_b200.adjoint import kappa_apply
    A, V, om, mesh = setup(sf, 3, 6, 4)
    nc, nq = mesh.cell_dof_ids.shape[0], om.SQ ** 3
    g = torch.Generator(device="cuda").manual_seed(0)
    x = (torch.rand(A.n, dtype=torch.float64, device="cuda", generator=g) * 2 - 1).requires_grad_()
    kappa = torch.from_numpy(kappa_field(1, nc, nq)).cuda().requires_grad_()
    yb = torch.rand(A.n, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    y = kappa_apply(A, x, kappa)
    (y * yb).sum().backward()
    dx = torch.rand(A.n, dtype=torch.float64, device="cuda", generator=g)
    dk = torch.rand(nc, nq, dtype=torch.float64, device="cuda", generator=g)
    with torch.no_grad():
        f0 = torch.dot(yb, kappa_apply(A, x, kappa))
        fx = torch.dot(yb, kappa_apply(A, x + dx, kappa)) - f0
        fk = torch.dot(yb, kappa_apply(A, x, kappa + dk)) - f0
    assert abs(fx.item() - torch.dot(x.grad, dx).item()) < 1e-11 * abs(fx.item())
    assert abs(fk.item() - torch.sum(kappa.grad * dk).item()) < 1e-11 * abs(fk.item())
    # forward value against the oracle's variable-coefficient apply
    y_ref = O.lazy_mul(om, mesh, x.detach().cpu().numpy(), kappa=kappa.detach().cpu().numpy())
    assert np.abs(y.detach().cpu().numpy() - y_ref).max() < 1e-12 * np.abs(y_ref).max()


def test_objective_gradient_fd_and_oracle(sf):
    import torch
    from ncihackaton2023_b200.adjoint import objective, objective_gradient
    p, deg, n = 3, 6, 3
    A, V, om, mesh = setup(sf, p, deg, n)
    nc, nq = mesh.cell_dof_ids.shape[0], om.SQ ** 3
    cq = O.cell_quantities(om, mesh)
    b = O.rhs(om, mesh, O.sin_forcing, cq)
    kappa_true = kappa_field(7, nc, nq)
    kappa = kappa_field(8, nc, nq)
    _, _, u_obs = O.adjoint_gradient_sparse(om, mesh, b, np.zeros(mesh.n_free), kappa_true, cq)
    J_ref, g_ref, _ = O.adjoint_gradient_sparse(om, mesh, b, u_obs, kappa, cq)
    bd, uo = torch.from_numpy(b).cuda(), torch.from_numpy(u_obs).cuda()
    kd = torch.from_numpy(kappa).cuda()
    J, g, u, info = objective_gradient(A, bd, uo, kd, reltol=1e-13)
    g = g.cpu().numpy()
    assert abs(J - J_ref) < 1e-9 * abs(J_ref)
    assert np.abs(g - g_ref).max() < 1e-8 * np.abs(g_ref).max()
    d = np.random.default_rng(9).normal(0, 1, (nc, nq))
    eps = 1e-6
    dd = torch.from_numpy(d).cuda()
    Jp = objective(A, bd, uo, kd + eps * dd, reltol=1e-13)
    Jm = objective(A, bd, uo, kd - eps * dd, reltol=1e-13)
    fd = (Jp - Jm) / (2 * eps)
    assert abs(fd - np.sum(g * d)) < 1e-5 * abs(fd)


def test_rrule_call_sequence(sf):
    """The C-ABI calls of the Julia ChainRulesCore.rrule binding: forward
    sf_set_coefficient_device + sf_apply; pullback sf_apply(ybar) for x and
    sf_kappa_vjp(x, ybar) for kappa. Checked against the torch autograd rule."""
    import ctypes as C

    import torch
    from ncihackaton2023_b200 import _lib
    from ncihackaton2023_b200.adjoint import kappa_apply
    A, V, om, mesh = setup(sf, 3, 6, 3, 0.2, 4)
    nc, nq = 27, 64
    lib = _lib.lib
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(8)
    kappa = torch.from_numpy(kappa_field(2, nc, nq)).cuda()
    x = torch.from_numpy(rng.uniform(-1, 1, A.n)).cuda()
    yb = torch.from_numpy(rng.uniform(-1, 1, A.n)).cuda()
    ptr = lambda t: C.c_void_p(t.data_ptr())
    # forward
    assert lib.sf_set_coefficient_device(A._h, ptr(kappa), s) == _lib.SF_OK
    y = torch.empty_like(x)
    assert lib.sf_apply(A._h, _lib.SF_F64, ptr(x), ptr(y), s) == _lib.SF_OK
    # pullback
    assert lib.sf_set_coefficient_device(A._h, ptr(kappa), s) == _lib.SF_OK
    xbar = torch.empty_like(x)
    assert lib.sf_apply(A._h, _lib.SF_F64, ptr(yb), ptr(xbar), s) == _lib.SF_OK
    kbar = torch.empty_like(kappa)
    assert lib.sf_kappa_vjp(A._h, _lib.SF_F64, ptr(x), ptr(yb), ptr(kbar), s) == _lib.SF_OK
    # the torch rule
    xt = x.clone().requires_grad_(True)
    kt = kappa.clone().requires_grad_(True)
    yt = kappa_apply(A, xt, kt)
    yt.backward(yb)
    tol = lambda ref: 1e-12 * ref.abs().max().item()
    assert (y - yt.detach()).abs().max().item() <= tol(yt.detach())
    assert (xbar - xt.grad).abs().max().item() <= tol(xt.grad)
    assert (kbar - kt.grad).abs().max().item() <= tol(kt.grad)
    # and the kappa pullback against the oracle's VJP
    kb_ref = O.kappa_vjp(om, mesh, x.cpu().numpy(), yb.cpu().numpy())
    assert np.abs(kbar.cpu().numpy() - kb_ref).max() < 1e-12 * np.abs(kb_ref).max()
