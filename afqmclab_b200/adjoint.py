"""torch.autograd wrapper of the engine's adjoint (afqmc_pl_adjoint).

`MixedEnergy.apply(t, chol, phiT_up, phiT_dn, ctx)` returns Re E, the mixed
local energy E = sum_w den_w E_w / sum_w den_w of a fixed walker population,
as a float64 scalar; its backward uses the engine's hand-written adjoint
(gradients with respect to the one-body matrix t, the Cholesky vectors and
the trial orbitals).  It exists to check the adjoint against finite
differences; the engine does the work on the GPU.
"""
import numpy as np
import torch

from . import capi
from .inputs import MoleculeInputs


class AdjointContext:
    """The fixed part of the evaluation: sizes, walkers, a template model."""

    def __init__(self, model: MoleculeInputs, walkers, seed=1):
        self.model = model
        self.wf, self.logw, self.alive = walkers
        self.seed = seed

    def evaluate(self, t, chol, phiT_up, phiT_dn, want_chol=True):
        m = self.model
        mm = MoleculeInputs(n=m.n, nup=m.nup, ndn=m.ndn, G=m.G, dt=m.dt,
                            t=np.asfortranarray(t), K=m.K, chol=np.asfortranarray(chol), bg=m.bg,
                            phiTUp=np.asfortranarray(phiT_up), phiTDn=np.asfortranarray(phiT_dn),
                            logwT=m.logwT)
        for name in ("Kp", "expMinusDtK", "expHalfDtK", "expMinusHalfDtK", "logwDt", "logwHalf",
                     "ET", "force_cap"):
            setattr(mm, name, getattr(m, name))
        eng = capi.pl_engine(mm, self.wf.shape[2], self.seed, precision=capi.AFQMC_FP64)
        try:
            eng.set_walkers(self.wf, self.logw, self.alive)
            return eng.adjoint(want_chol=want_chol)
        finally:
            eng.close()


class MixedEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, t, chol, phiT_up, phiT_dn, actx):
        out = actx.evaluate(t.detach().cpu().numpy(), chol.detach().cpu().numpy(),
                            phiT_up.detach().cpu().numpy(), phiT_dn.detach().cpu().numpy())
        ctx.grads = (out["dE_dt"], out["dE_dchol"], out["dE_dconj_phiT"][0],
                     out["dE_dconj_phiT"][1])
        return torch.tensor(float(np.real(out["E"])), dtype=torch.float64)

    @staticmethod
    def backward(ctx, g):
        dt, dc, du, dd = ctx.grads
        # real inputs: d Re(E)/dx = Re(dE/dx); complex orbitals: torch's
        # gradient of a real output is 2 d/dconj(z) of it = dE/dconj(z),
        # since E depends on conj(phiT) only
        return (g * torch.from_numpy(np.real(dt).copy()), g * torch.from_numpy(np.real(dc).copy()),
                g * torch.from_numpy(du.copy()), g * torch.from_numpy(dd.copy()), None)
