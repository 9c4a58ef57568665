"""The adjoint gradient behind a torch.autograd.Function: the misfit of a
run's receiver output as a differentiable function of per-cell
log-conductivity.  torch is the harness here; the forward run and the
gradient are the library's CUDA path (temf_run with recording, then
temf_adjoint).  Marked ``gpu``; run on a B200."""
import numpy as np
import pytest
import torch

from temf3dt_b200 import fetd
from tests.golden_cases import cell_grid_2x2x2, small_synth, synth_oracle_model

pytestmark = pytest.mark.gpu


class Misfit(torch.autograd.Function):
    """J(m) = 1/2 sum w (d(m) - d_obs)^2 over the dBz/dt column, with
    sigma_t = exp(m_cell(t)) inside the inversion cells and the background
    conductivity elsewhere.  The runs replay the observed run's accept/reject
    decisions, so every output row stays at the observed row's time."""

    @staticmethod
    def forward(ctx, m, case):
        g, model, sig0, mu, cell, d_obs, w, forced = case
        sig = sig0.copy()
        inside = cell >= 0
        sig[inside] = np.exp(m.detach().cpu().numpy()[cell[inside]])
        g.set_media(sig, mu)
        g.assemble()
        g.adjoint_record(50)
        c = model.ctl
        out = g.run(c.sp_division, c.sp_double, c.sp_dblesize, c.time_maximum, forced=forced)
        r = out.fields - d_obs
        ctx.case = case
        ctx.dJ = w * r
        ctx.ncell = m.numel()
        return torch.tensor(0.5 * float(np.sum(w * r * r)), dtype=torch.float64)

    @staticmethod
    def backward(ctx, gJ):
        g = ctx.case[0]
        grad, _, _ = g.adjoint(ctx.dJ, ctx.case[4], ctx.ncell)
        g.adjoint_record(0)
        return gJ * torch.from_numpy(grad), None


def test_autograd_gradient_descends_the_misfit():
    model = small_synth()
    om = synth_oracle_model(model)
    cell = cell_grid_2x2x2(om)
    with fetd.FetdGPU(0) as g:
        info = fetd.load_case(g, model.mesh, model.ctl)
        sig0, mu = info["sig"], info["mu"]
        # observed data: cell 3 twice as conductive; dBz/dt weighted by 1/max^2
        sig_true = sig0.copy()
        sig_true[cell == 3] *= 2.0
        g.set_media(sig_true, mu)
        g.assemble()
        c = model.ctl
        obs = g.run(c.sp_division, c.sp_double, c.sp_dblesize, c.time_maximum)
        d_obs = obs.fields
        w = np.zeros_like(d_obs)
        w[:, :, 5] = 1.0 / np.abs(d_obs[:, :, 5]).max() ** 2
        case = (g, model, sig0, mu, cell, d_obs, w, obs.trial_accepted.astype(np.int32))
        m = torch.full((8,), float(np.log(sig0[cell >= 0][0])), dtype=torch.float64, requires_grad=True)
        J0 = Misfit.apply(m, case)
        J0.backward()
        grad = m.grad.clone()
        assert torch.isfinite(grad).all() and grad.abs().max() > 0
        # raising the perturbed cell's conductivity lowers the misfit
        assert float(grad[3]) < 0
        # directional derivative along steepest descent by central differences
        d = -grad / grad.norm()
        eps = 1e-3
        with torch.no_grad():
            Jp = float(Misfit.apply(m + eps * d, case))
            Jm = float(Misfit.apply(m - eps * d, case))
        fd = (Jp - Jm) / (2 * eps)
        assert fd < 0
        assert abs(fd - float(grad @ d)) <= 1e-3 * abs(fd), (fd, float(grad @ d))
        g.adjoint_record(0)
