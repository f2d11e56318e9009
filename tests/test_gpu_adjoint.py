"""GPU adjoint (sp_adjoint_rk4) against the oracle's discrete adjoint and
central finite differences; torch.autograd wrapper."""
import numpy as np
import pytest
import torch

from ics import gaussian_noise, rel_l2

pytestmark = pytest.mark.gpu


def forward(sp, n, q0, pars, dt, steps):
    nu0, cx, cy, cz = pars
    conv = sp.Convection(n, n, n, 1.0 / n, nu0, 0.0, cx, cy, cz)
    f0, f1 = conv.field(), conv.field()
    conv.upload(f0, q0)
    conv.DoRK4(f0, f1, 0.0, dt, steps)
    return conv.download(f1)


def J_of(sp, n, q0, qt, pars, dt, steps):
    q = forward(sp, n, q0, pars, dt, steps)
    return 0.5 * ((q - qt) ** 2).sum()


def central_difference(sp, n, q0, qt, pars, dq, dp, h, dt, steps):
    """(J(+h) - J(-h)) / 2h for J = 0.5||q_n - qt||^2, evaluated as
    sum (q+ - q-)(q+ + q- - 2 qt) / 4h so that J's leading digits do not cancel."""
    qp = forward(sp, n, q0 + h * dq, tuple(np.add(pars, h * dp)), dt, steps)
    qm = forward(sp, n, q0 - h * dq, tuple(np.subtract(pars, h * dp)), dt, steps)
    return float(((qp - qm) * (qp + qm - 2 * qt)).sum() / (4 * h))


def test_adjoint_matches_oracle_and_checkpointing(sp, orc):
    from stencilparareal_b200.adjoint import misfit_gradient
    n, steps, dt = 12, 9, 2e-3
    pars = (0.05, 0.7, -0.4, 0.3)
    conv = sp.Convection(n, n, n, 1.0 / n, *pars[:1], 0.0, *pars[1:])
    q0 = gaussian_noise(n, seed=5, amp=1e-2)
    qt = gaussian_noise(n, seed=6, amp=1e-2) * 0.9
    f0, ft = conv.field(), conv.field()
    conv.upload(f0, q0)
    conv.upload(ft, qt)
    Jo, go, gpo = orc.adjoint_rk4(orc.params(n, nu0=pars[0], cx=pars[1], cy=pars[2], cz=pars[3]), q0, qt, 0.0, dt,
                                  steps)
    grads = []
    for ck in (1, 3, 0, steps):
        J, g, gp = misfit_gradient(conv, f0, ft, 0.0, dt, steps, checkpoint_every=ck)
        gq = conv.download(g)
        assert abs(J - Jo) <= 1e-12 * abs(Jo)
        assert rel_l2(gq, go) < 1e-11
        np.testing.assert_allclose(gp, gpo, rtol=1e-9, atol=1e-12)
        grads.append(gq)
    for gq in grads[1:]:
        assert rel_l2(gq, grads[0]) < 1e-14


def test_adjoint_vs_central_differences_small(sp):
    from stencilparareal_b200.adjoint import misfit_gradient
    n, steps, dt = 16, 20, 1e-3
    pars = (0.02, 1.0, 0.5, 0.25)
    q0 = gaussian_noise(n, seed=1, amp=1e-2)
    qt = gaussian_noise(n, seed=2, amp=1e-2)
    conv = sp.Convection(n, n, n, 1.0 / n, pars[0], 0.0, *pars[1:])
    f0, ft = conv.field(), conv.field()
    conv.upload(f0, q0)
    conv.upload(ft, qt)
    J, g, gp = misfit_gradient(conv, f0, ft, 0.0, dt, steps)
    gq = conv.download(g)
    rng = np.random.default_rng(4)
    h = 1e-6
    for _ in range(4):
        dq = rng.standard_normal(q0.shape)
        dp = rng.standard_normal(4)
        nrm = np.sqrt((dq ** 2).sum() + (dp ** 2).sum())
        dq, dp = dq / nrm, dp / nrm
        fd = central_difference(sp, n, q0, qt, pars, dq, dp, h, dt, steps)
        ad = (gq * dq).sum() + np.dot(gp, dp)
        assert abs(fd - ad) <= 1e-6 * max(abs(fd), 1e-12), (fd, ad)


def test_autograd_function(sp):
    from stencilparareal_b200.adjoint import rk4_propagate
    n, steps, dt = 12, 6, 2e-3
    q0 = torch.tensor(gaussian_noise(n, seed=7, amp=1e-2), device="cuda", requires_grad=True)
    params = torch.tensor([0.03, 0.9, -0.2, 0.4], dtype=torch.float64, requires_grad=True)
    qt = torch.tensor(gaussian_noise(n, seed=8, amp=1e-2), device="cuda")
    qn = rk4_propagate(q0, params, 1.0 / n, 0.0, dt, steps)
    loss = 0.5 * ((qn - qt) ** 2).sum()
    loss.backward()
    # the same quantities through the C ABI misfit entry point
    from stencilparareal_b200.adjoint import misfit_gradient
    conv = sp.Convection(n, n, n, 1.0 / n, 0.03, 0.0, 0.9, -0.2, 0.4)
    f0, ft = conv.field(), conv.field()
    conv.upload(f0, q0.detach().cpu().numpy())
    conv.upload(ft, qt.cpu().numpy())
    J, g, gp = misfit_gradient(conv, f0, ft, 0.0, dt, steps)
    assert abs(loss.item() - J) <= 1e-12 * J
    assert rel_l2(q0.grad.cpu().numpy(), conv.download(g)) < 1e-13
    np.testing.assert_allclose(params.grad.numpy(), gp, rtol=1e-12, atol=0)


def test_adjoint_128cube_400_steps_vs_central_differences(sp):
    """Gradient of 0.5||q(T)-q_target||^2 wrt q0, nu, c through 400 RK4 FP64 steps (dt=5e-5) at 128^3,
    checkpoint every 20 steps, against central differences on 16 random unit directions in (q0, nu, c).

    With h=1e-6 the central difference carries an absolute FP64 noise of ~1e-9 (two 400-step runs
    whose difference is ~1e-6 of the fields); measured against the gradient norm (the directions are
    unit vectors) the adjoint agrees to < 1e-6.  J is exactly quadratic in q0, so h=1e-4 removes that
    noise and the per-direction relative agreement is < 1e-6 as well."""
    from stencilparareal_b200.adjoint import misfit_gradient
    n, steps, dt = 128, 400, 5e-5
    pars = (0.01, 1.0, 1.0, 1.0)
    q0 = gaussian_noise(n, seed=0)
    rng3 = np.random.default_rng(3)
    conv = sp.Convection(n, n, n, 1.0 / n, pars[0], 0.0, *pars[1:])
    f0, ft, fp = conv.field(), conv.field(), conv.field()
    conv.upload(fp, q0 + 1e-2 * rng3.uniform(-1, 1, size=q0.shape))
    conv.DoRK4(fp, ft, 0.0, dt, steps)  # q_target: forward solve from the perturbed q0
    conv.upload(f0, q0)
    J, g, gp = misfit_gradient(conv, f0, ft, 0.0, dt, steps, checkpoint_every=20)
    gq = conv.download(g)
    qt = conv.download(ft)
    gnorm = np.sqrt((gq ** 2).sum() + np.dot(gp, gp))
    rng = np.random.default_rng(4)
    worst_norm, worst_rel = 0.0, 0.0
    for _ in range(16):
        dq = rng.standard_normal(q0.shape)
        dp = rng.standard_normal(4)
        nrm = np.sqrt((dq ** 2).sum() + (dp ** 2).sum())
        dq, dp = dq / nrm, dp / nrm
        ad = (gq * dq).sum() + np.dot(gp, dp)
        fd6 = central_difference(sp, n, q0, qt, pars, dq, dp, 1e-6, dt, steps)
        fd4 = central_difference(sp, n, q0, qt, pars, dq, dp, 1e-4, dt, steps)
        worst_norm = max(worst_norm, abs(fd6 - ad) / gnorm)
        worst_rel = max(worst_rel, abs(fd4 - ad) / abs(fd4))
    print(f"adjoint 128^3: J={J:.6e} |grad|={gnorm:.4e}; h=1e-6: max |fd-ad|/|grad| = {worst_norm:.3e}; "
          f"h=1e-4: max |fd-ad|/|fd| = {worst_rel:.3e}")
    assert worst_norm < 1e-6, worst_norm
    assert worst_rel < 1e-6, worst_rel
