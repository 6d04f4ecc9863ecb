"""IMPT spot-weight optimisation on the device, with checkpoint / resume.

The reference has no optimiser: its only affordance is calling
``proton_raytrace_cuda`` once per beam and ``proton_spot_cuda`` per weight
change (plan_impt.py:148-155).  Here the WET stays resident, the dose of a
weight vector is the pencil-beam kernel (``ProtonBeamPlan.dose``) and its
gradient the hand-written adjoint kernel D^T g (``ProtonBeamPlan.adjoint``)
behind ``torch.autograd`` (``engine.proton_dose_autograd``).

* ``DoseObjective``: a sum of quadratic voxel terms in float64 -- uniform
  dose, maximum dose (only the overdose counts), minimum dose (only the
  underdose counts) -- over voxel sets held as flat index tensors, so that an
  evaluation never synchronises with the host.
* ``ImptOptimizer``: projected Adam on the spot weights (weights >= 0 after
  every step); ``save``/``load`` write and restore the weights, Adam's moments
  and step count and the iteration, so an interrupted run continues exactly.
  With ``voxels="objective"`` every step computes the dose and the adjoint
  at the objective's voxels only (``ProtonBeamPlan.dose_list`` /
  ``adjoint_list``): the objective and its gradient depend on nothing else,
  and target plus organs at risk are a small part of the grid.
* ``ImrtOptimizer``: the same loop on the segment (control-point) weights of
  photon beams, through ``engine.PhotonPlanBasis`` and its adjoint kernel.
* ``FluenceOptimizer``: the same loop on beamlet fluence maps of photon
  control points, through ``engine.PhotonFluenceBeam`` (TERMA modulated by
  the map, CCCS forward, the hand-written CCCS transpose backward).
* ``save_influence_csr``/``load_influence_csr``: a dose-influence matrix
  (``ProtonBeamPlan.influence_csr``) cached as ``.npz``."""
from __future__ import annotations

import os

import numpy as np
import torch

from . import engine


class DoseObjective:
    """f(D) = sum_k w_k sum_{v in V_k} r_k(D_v)^2, evaluated in float64, with
    r = D - d (uniform), max(D - d, 0) (maximum dose) or min(D - d, 0)
    (minimum dose)."""

    KINDS = ("uniform", "max", "min")

    def __init__(self):
        self.terms = []
        self._union = None
        self._pos = None

    @staticmethod
    def _index(mask: torch.Tensor) -> torch.Tensor:
        if mask.dtype != torch.bool:
            raise ValueError("a voxel set is a boolean mask of the dose grid")
        return torch.nonzero(mask.reshape(-1), as_tuple=False).squeeze(1)

    def add(self, kind: str, mask: torch.Tensor, dose: float, weight: float = 1.0) -> "DoseObjective":
        if kind not in self.KINDS:
            raise ValueError("term kind must be one of %s" % (self.KINDS,))
        if weight < 0:
            raise ValueError("term weights must be non-negative")
        self.terms.append((kind, self._index(mask), float(dose), float(weight), tuple(mask.shape)))
        return self

    def uniform(self, mask, dose, weight=1.0):
        return self.add("uniform", mask, dose, weight)

    def max_dose(self, mask, dose, weight=1.0):
        return self.add("max", mask, dose, weight)

    def min_dose(self, mask, dose, weight=1.0):
        return self.add("min", mask, dose, weight)

    def voxel_union(self) -> torch.Tensor:
        """Sorted flat indices of every voxel some term reads (the only
        voxels whose dose the objective depends on)."""
        if self._pos is None or len(self._pos) != len(self.terms):
            if not self.terms:
                raise ValueError("the objective has no terms")
            self._union = torch.unique(torch.cat([t[1] for t in self.terms]))
            self._pos = [torch.searchsorted(self._union, t[1]) for t in self.terms]
        return self._union

    def on_list(self, dose_list: torch.Tensor) -> torch.Tensor:
        """The objective from the dose at voxel_union() only (same terms,
        same float64 arithmetic as __call__)."""
        self.voxel_union()
        f = torch.zeros((), dtype=torch.float64, device=dose_list.device)
        for (kind, _, d, w, _), pos in zip(self.terms, self._pos):
            r = dose_list.index_select(0, pos).double() - d
            if kind == "max":
                r = torch.clamp(r, min=0.0)
            elif kind == "min":
                r = torch.clamp(r, max=0.0)
            f = f + w * (r * r).sum()
        return f

    def __call__(self, dose: torch.Tensor) -> torch.Tensor:
        flat = dose.reshape(-1)
        f = torch.zeros((), dtype=torch.float64, device=dose.device)
        for kind, idx, d, w, shape in self.terms:
            if tuple(dose.shape) != shape:
                raise ValueError("dose has shape %s, the objective's voxel sets %s" % (tuple(dose.shape), shape))
            r = flat.index_select(0, idx).double() - d
            if kind == "max":
                r = torch.clamp(r, min=0.0)
            elif kind == "min":
                r = torch.clamp(r, max=0.0)
            f = f + w * (r * r).sum()
        return f


class ImptOptimizer:
    """Projected Adam on the spot weights of one or more beams of a plan.

    ``plans``: ``engine.ProtonBeamPlan`` per beam (or any object with the same
    ``dose``/``adjoint``/``n_spots``/``mu``); ``wets``: each beam's smoothed WET
    on the dose grid.  The weight vector concatenates the beams' spots in
    order; ``lr`` defaults to ``lr_frac`` x the mean initial weight."""

    def __init__(self, plans, wets, objective: DoseObjective, mu: torch.Tensor | None = None, lr: float | None = None,
                 lr_frac: float = 0.02, voxels: str = "volume"):
        self.plans, self.wets = list(plans), list(wets)
        if len(self.plans) != len(self.wets) or not self.plans:
            raise ValueError("one WET volume per beam is required")
        self.objective = objective
        self.sizes = [int(p.n_spots) for p in self.plans]
        mu0 = torch.cat([p.mu for p in self.plans]) if mu is None else mu
        if mu0.numel() != sum(self.sizes):
            raise ValueError("mu must hold one weight per spot of all beams")
        self.mu = mu0.detach().to(device=self.wets[0].device, dtype=torch.float32).clone().requires_grad_(True)
        self.lr = float(lr) if lr is not None else float(lr_frac * self.mu.detach().mean().item())
        self.opt = torch.optim.Adam([self.mu], lr=self.lr)
        self.iteration = 0
        self.value = None  # objective (device tensor) at the weights before the last step
        if voxels not in ("volume", "objective"):
            raise ValueError("voxels must be 'volume' or 'objective'")
        # "objective": each step evaluates the dose and its adjoint at the
        # objective's voxels only (the voxel-list kernels), which gives the
        # same objective and gradient for a fraction of the work
        self.voxels = voxels
        self._list = objective.voxel_union().to(torch.int32) if voxels == "objective" else None

    def dose(self, mu: torch.Tensor | None = None) -> torch.Tensor:
        """Total dose of all beams; differentiable in ``mu`` (default: the
        current weights)."""
        m = self.mu if mu is None else mu
        parts = torch.split(m, self.sizes)
        total = None
        for q, w, p in zip(parts, self.wets, self.plans):
            d = engine.proton_dose_autograd(q.contiguous(), w, p)
            total = d if total is None else total + d
        return total

    def dose_list(self, mu: torch.Tensor | None = None) -> torch.Tensor:
        """Total dose at the objective's voxels (``objective.voxel_union()``);
        differentiable in ``mu``."""
        m = self.mu if mu is None else mu
        vox = self._list if self._list is not None else self.objective.voxel_union().to(torch.int32)
        parts = torch.split(m, self.sizes)
        total = None
        for q, w, p in zip(parts, self.wets, self.plans):
            d = engine.proton_dose_list_autograd(q.contiguous(), w, p, vox)
            total = d if total is None else total + d
        return total

    def _objective(self, mu: torch.Tensor) -> torch.Tensor:
        if self.voxels == "objective":
            return self.objective.on_list(self.dose_list(mu))
        return self.objective(self.dose(mu))

    def evaluate(self) -> float:
        with torch.no_grad():
            return float(self._objective(self.mu.detach()))

    def scale_to(self, mask: torch.Tensor, dose: float) -> float:
        """Scales the weights so that the mean dose over ``mask`` is ``dose``
        (before the first step only); returns the factor."""
        if self.iteration:
            raise RuntimeError("scale_to is for the initial weights")
        with torch.no_grad():
            d = self.dose(self.mu.detach()).double()
            mean = float(d.reshape(-1)[mask.reshape(-1)].mean())
            if not mean > 0:
                raise ValueError("the initial weights give no dose in the mask")
            k = dose / mean
            self.mu.mul_(k)
        self.lr = self.lr * k
        for g in self.opt.param_groups:
            g["lr"] = self.lr
        return k

    def step(self):
        """One iteration: dose, objective, adjoint gradient, Adam, projection
        onto mu >= 0.  Does not synchronise with the host."""
        self.opt.zero_grad(set_to_none=True)
        f = self._objective(self.mu)
        f.backward()
        self.opt.step()
        with torch.no_grad():
            self.mu.clamp_(min=0.0)
        self.value = f.detach()
        self.iteration += 1

    def run(self, iterations: int, checkpoint: str | None = None, every: int | None = None, log=None):
        """``iterations`` steps; with ``checkpoint``, the state is saved every
        ``every`` iterations (default: at the end only) and at the end."""
        for _ in range(int(iterations)):
            self.step()
            if log and self.iteration % 50 == 0:
                log("iteration %d objective %.6g" % (self.iteration, float(self.value)))
            if checkpoint and every and self.iteration % every == 0:
                self.save(checkpoint)
        if checkpoint:
            self.save(checkpoint)

    # -- checkpoint / resume --------------------------------------------------
    def state_dict(self) -> dict:
        return {"version": 1, "mu": self.mu.detach().cpu().clone(), "adam": self.opt.state_dict(),
                "iteration": self.iteration, "sizes": list(self.sizes), "lr": self.lr}

    def load_state_dict(self, sd: dict):
        if sd.get("version") != 1:
            raise ValueError("unsupported optimiser checkpoint")
        if list(sd["sizes"]) != self.sizes:
            raise ValueError("checkpoint was written for beams of %s weights, this plan has %s" %
                             (list(sd["sizes"]), self.sizes))
        with torch.no_grad():
            self.mu.copy_(sd["mu"].to(self.mu.device))
        self.opt.load_state_dict(sd["adam"])
        self.lr = float(sd["lr"])
        self.iteration = int(sd["iteration"])

    def save(self, path: str):
        """Written to a temporary file and renamed: an interrupted write
        leaves the previous checkpoint intact."""
        tmp = str(path) + ".tmp"
        torch.save(self.state_dict(), tmp)
        os.replace(tmp, str(path))

    def load(self, path: str):
        self.load_state_dict(torch.load(str(path), map_location="cpu", weights_only=True))


class ImrtOptimizer(ImptOptimizer):
    """Projected Adam on the segment (control-point) weights of photon beams.

    ``bases``: one ``engine.PhotonPlanBasis`` per beam; the plan dose for
    weights w is sum over beams of ``engine.photon_dose_autograd(w_beam,
    basis)`` (the basis combination forward, the hand-written adjoint kernel
    backward), and w = 1 is the plan as delivered (the control-point loop's
    dose bit for bit).  The loop, the objective, ``scale_to``, checkpoint and
    resume are ``ImptOptimizer``'s."""

    def __init__(self, bases, objective: DoseObjective, weights: torch.Tensor | None = None,
                 lr: float | None = None, lr_frac: float = 0.02):
        self.plans = list(bases)
        if not self.plans:
            raise ValueError("at least one photon beam basis is required")
        self.wets = [None] * len(self.plans)
        self.objective = objective
        self.sizes = [int(b.n) for b in self.plans]
        dev = self.plans[0].device
        w0 = torch.ones(sum(self.sizes), dtype=torch.float32, device=dev) if weights is None else weights
        if w0.numel() != sum(self.sizes):
            raise ValueError("weights must hold one value per control point of all beams")
        self.mu = w0.detach().to(device=dev, dtype=torch.float32).clone().requires_grad_(True)
        self.lr = float(lr) if lr is not None else float(lr_frac * self.mu.detach().mean().item())
        self.opt = torch.optim.Adam([self.mu], lr=self.lr)
        self.iteration = 0
        self.value = None
        self.voxels = "volume"
        self._list = None

    def dose(self, mu: torch.Tensor | None = None) -> torch.Tensor:
        """Plan dose of all beams for segment weights ``mu`` (default: the
        current weights); differentiable."""
        m = self.mu if mu is None else mu
        total = None
        for q, basis in zip(torch.split(m, self.sizes), self.plans):
            d = engine.photon_dose_autograd(q.contiguous(), basis)
            total = d if total is None else total + d
        return total

    def dose_list(self, mu=None):
        raise NotImplementedError("segment weights are optimised on the full volume")


class FluenceOptimizer(ImptOptimizer):
    """Projected Adam on the beamlet fluence maps of photon control points.

    ``beams``: one ``engine.PhotonFluenceBeam`` per control point (its TERMA
    computed once); ``output_factors`` (default 1) scale each control point's
    dose as the plan loop does (plan_imrt.py:151-153).  The plan dose for maps
    F is sum_b OF_b D_b(F_b), differentiable through
    ``engine.photon_fluence_dose_autograd`` (modulated TERMA + CCCS forward,
    the CCCS transpose backward); F = 1 is the plan as delivered.  Maps are
    kept >= 0 after every step.  The loop, the objective, ``scale_to``,
    checkpoint and resume are ``ImptOptimizer``'s."""

    def __init__(self, beams, objective: DoseObjective, output_factors=None, fluence: torch.Tensor | None = None,
                 lr: float | None = None, lr_frac: float = 0.02):
        self.plans = list(beams)
        if not self.plans:
            raise ValueError("at least one control point is required")
        self.wets = [None] * len(self.plans)
        self.objective = objective
        self.sizes = [int(b.na * b.nb) for b in self.plans]
        of = [1.0] * len(self.plans) if output_factors is None else [float(x) for x in output_factors]
        if len(of) != len(self.plans):
            raise ValueError("one output factor per control point is required")
        self.output_factors = of
        dev = self.plans[0].device
        f0 = torch.ones(sum(self.sizes), dtype=torch.float32, device=dev) if fluence is None else fluence
        if f0.numel() != sum(self.sizes):
            raise ValueError("fluence must hold one value per beamlet of all control points")
        self.mu = f0.detach().to(device=dev, dtype=torch.float32).clone().requires_grad_(True)
        self.lr = float(lr) if lr is not None else float(lr_frac * self.mu.detach().mean().item())
        self.opt = torch.optim.Adam([self.mu], lr=self.lr)
        self.iteration = 0
        self.value = None
        self.voxels = "volume"
        self._list = None

    def dose(self, mu: torch.Tensor | None = None) -> torch.Tensor:
        """Plan dose for fluence maps ``mu`` (default: the current maps, all
        control points' beamlets concatenated); differentiable."""
        m = self.mu if mu is None else mu
        total = None
        for q, beam, of in zip(torch.split(m, self.sizes), self.plans, self.output_factors):
            d = engine.photon_fluence_dose_autograd(q.reshape(beam.nb, beam.na), beam)
            d = d * of if of != 1.0 else d
            total = d if total is None else total + d
        return total

    def dose_list(self, mu=None):
        raise NotImplementedError("fluence maps are optimised on the full volume")


def save_influence_csr(path: str, row_ptr: torch.Tensor, col: torch.Tensor, val: torch.Tensor, shape, n_spots: int):
    """Caches a dose-influence matrix (voxel rows of ``shape``, ``n_spots``
    columns) as ``.npz``."""
    n_vox = int(np.prod(shape))
    if row_ptr.numel() != n_vox + 1 or col.numel() != val.numel():
        raise ValueError("inconsistent CSR arrays")
    np.savez(path, row_ptr=row_ptr.cpu().numpy(), col=col.cpu().numpy(), val=val.cpu().numpy(),
             shape=np.asarray(shape, np.int64), n_spots=np.int64(n_spots))


def load_influence_csr(path: str, device="cuda"):
    """(row_ptr, col, val, shape, n_spots) of a cached influence matrix."""
    with np.load(path) as z:
        row_ptr, col, val = (torch.as_tensor(z[k]).to(device) for k in ("row_ptr", "col", "val"))
        shape = tuple(int(v) for v in z["shape"])
        n_spots = int(z["n_spots"])
    if row_ptr.dtype != torch.int64 or col.dtype != torch.int32 or val.dtype != torch.float32:
        raise ValueError("influence matrix arrays have unexpected types")
    if row_ptr.numel() != int(np.prod(shape)) + 1 or int(row_ptr[-1]) != col.numel():
        raise ValueError("influence matrix arrays are inconsistent")
    return row_ptr, col, val, shape, n_spots
