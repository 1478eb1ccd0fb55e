"""Resistivity tomography on the GPU: misfit and adjoint gradient (torch.autograd) against the
float64 sparse-direct oracle, and against central finite differences (eps = 1e-4) of the GPU
misfit on 20 random cells."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(hfm):
    import torch
    tm = hfm.tomography
    n = 16
    survey = tm.make_survey(n=n, n_src=4, n_rec=12, seed=3)
    solver = tm.ForwardSolver(n, group=4, tol=1e-10)
    sig_true = tm.true_sigma(n, seed=3)
    d_obs = tm.observe(sig_true, survey, solver)
    yield hfm, torch, tm, survey, solver, d_obs
    solver.close()


def test_gradient_matches_float64_oracle(setup):
    hfm, torch, tm, survey, solver, d_obs = setup
    from oracle import tomography as otomo
    n = survey.n
    logs = torch.zeros((3, n, n, n), dtype=torch.float64, device="cuda", requires_grad=True)
    J = tm.misfit(logs, survey, d_obs, solver)
    J.backward()
    g = logs.grad.cpu().numpy()
    sig = np.ones((3, n, n, n))
    Jr, gr, _ = otomo.misfit(sig, survey.q.double().cpu().numpy(), survey.receivers.cpu().numpy(),
                             d_obs.cpu().numpy())
    assert float(J.detach()) == pytest.approx(Jr, rel=1e-7)
    err = np.abs(g - gr).max() / np.abs(gr).max()
    assert err < 1e-6, err


def test_checkpointed_and_recomputed_backward_agree(setup):
    hfm, torch, tm, survey, solver, d_obs = setup
    n = survey.n
    grads = []
    for recompute in (False, True):
        logs = torch.full((3, n, n, n), 0.1, dtype=torch.float64, device="cuda", requires_grad=True)
        tm.misfit(logs, survey, d_obs, solver, recompute=recompute).backward()
        grads.append(logs.grad.clone())
    assert float((grads[0] - grads[1]).abs().max() / grads[0].abs().max()) < 1e-7


def test_gradient_matches_finite_differences(setup):
    hfm, torch, tm, survey, solver, d_obs = setup
    n = survey.n
    logs = torch.zeros((3, n, n, n), dtype=torch.float64, device="cuda", requires_grad=True)
    tm.misfit(logs, survey, d_obs, solver).backward()
    g = logs.grad.cpu().numpy()
    gmax = np.abs(g).max()
    rng = np.random.default_rng(11)
    eps = 1e-4
    base = logs.detach().clone()
    for _ in range(20):
        k, z, y, x = (int(rng.integers(0, 3)),) + tuple(int(v) for v in rng.integers(0, n, 3))
        lp, lm = base.clone(), base.clone()
        lp[k, z, y, x] += eps
        lm[k, z, y, x] -= eps
        fd = (tm.misfit_value(lp, survey, d_obs, solver) - tm.misfit_value(lm, survey, d_obs, solver)) / (2 * eps)
        # float32 conductivities: exp(+-eps) is rounded to float32 (relative 6e-8 on a 1e-4 step)
        assert abs(fd - g[k, z, y, x]) <= 2e-3 * abs(g[k, z, y, x]) + 1e-4 * gmax, (k, z, y, x, fd, g[k, z, y, x])
