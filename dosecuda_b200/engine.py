"""Device-resident interface of the dose engines.

Inputs and outputs are torch CUDA tensors (float32, C-contiguous, shape
(nz, ny, nx)); work is enqueued on the current torch stream of the tensor's
device (or the stream given) and the call returns without synchronising.
torch is used for device memory and streams only; the compute is
libdosecuda.so.

    wet  = engine.proton_wet(rlsp, grid, beam, model)
    dose = engine.proton_dose(wet, grid, beam, engine.ProtonModelDevice(model))
    dose = engine.photon_dose(density, grid, model, cp)

``grid`` is any object with ``spacing`` and ``origin`` (e.g. a DoseGrid).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .dose_kernels import ControlPointView, PhotonModelView


def _check_volume(t: torch.Tensor, name: str):
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and t.dim() == 3):
        raise ValueError("'%s' must be a 3-dimensional float32 CUDA tensor." % name)
    if not t.is_contiguous():
        raise ValueError("'%s' must be C-contiguous." % name)


def _stream(t: torch.Tensor, stream):
    s = stream if stream is not None else torch.cuda.current_stream(t.device)
    return C.c_void_p(s.cuda_stream)


def _spacing(grid):
    sp = np.asarray(grid.spacing, dtype=np.float32)
    return _lib.f3((sp[0], sp[0], sp[0])) if sp.size == 1 else _lib.f3(sp)


def _out(like: torch.Tensor, out):
    if out is None:
        return torch.empty_like(like)
    _check_volume(out, "out")
    if out.shape != like.shape or out.device != like.device:
        raise ValueError("'out' must match the input volume's shape and device.")
    return out


def proton_wet(rlsp: torch.Tensor, grid, beam, model, out=None, stream=None) -> torch.Tensor:
    """Smoothed WET (cm) of every voxel for one proton beam."""
    _check_volume(rlsp, "rlsp")
    out = _out(rlsp, out)
    nz, ny, nx = rlsp.shape
    rc = _lib.load().dc_proton_raytrace_dev(
        rlsp.device.index, C.c_void_p(rlsp.data_ptr()), nz, ny, nx, _spacing(grid), _lib.f3(grid.origin),
        _lib.f3(beam.iso), float(beam.gantry_angle), float(beam.couch_angle), float(model.VSADX),
        float(model.VSADY), C.c_void_p(out.data_ptr()), _stream(rlsp, stream))
    _lib.raise_for(rc)
    return out


class ProtonModelDevice:
    """A proton beam model with its depth-dose tables resident on a device."""

    def __init__(self, model, device="cuda"):
        self.model = model
        self.VSADX = float(model.VSADX)
        self.VSADY = float(model.VSADY)
        self.divergence_params = np.ascontiguousarray(model.divergence_params, dtype=np.float32)
        self.lut_depths = torch.as_tensor(np.ascontiguousarray(model.lut_depths), device=device)
        self.lut_sigmas = torch.as_tensor(np.ascontiguousarray(model.lut_sigmas), device=device)
        self.lut_idds = torch.as_tensor(np.ascontiguousarray(model.lut_idds), device=device)
        self.n_energies, self.lut_len = self.lut_depths.shape


def proton_dose(wet: torch.Tensor, grid, beam, dmodel: ProtonModelDevice, out=None, stream=None,
                spots=None) -> torch.Tensor:
    """Pencil-beam dose of ``beam.spot_list`` (or ``spots``) from a smoothed WET."""
    _check_volume(wet, "wet")
    out = _out(wet, out)
    sp = np.ascontiguousarray(beam.spot_list if spots is None else spots, dtype=np.float32).reshape(-1, 4)
    nz, ny, nx = wet.shape
    rc = _lib.load().dc_proton_spot_dev(
        wet.device.index, C.c_void_p(wet.data_ptr()), nz, ny, nx, _spacing(grid), _lib.f3(grid.origin),
        _lib.f3(beam.iso), float(beam.gantry_angle), float(beam.couch_angle), dmodel.VSADX, dmodel.VSADY,
        dmodel.divergence_params.ctypes.data_as(C.c_void_p),
        dmodel.n_energies, dmodel.divergence_params.shape[1], C.c_void_p(dmodel.lut_depths.data_ptr()),
        C.c_void_p(dmodel.lut_sigmas.data_ptr()), C.c_void_p(dmodel.lut_idds.data_ptr()), dmodel.lut_len,
        sp.ctypes.data_as(C.c_void_p), sp.shape[0], C.c_void_p(out.data_ptr()), _stream(wet, stream))
    _lib.raise_for(rc)
    return out


def photon_dose(density: torch.Tensor, grid, model, cp, out=None, stream=None, views=None) -> torch.Tensor:
    """Collapsed-cone dose of one control point (before the output factor).
    ``views`` = (PhotonModelView, ControlPointView) may be passed to reuse the
    packed parameter blocks across calls."""
    _check_volume(density, "density")
    out = _out(density, out)
    mv, cv = views if views is not None else (PhotonModelView(model), ControlPointView(cp))
    nz, ny, nx = density.shape
    rc = _lib.load().dc_photon_dose_dev(
        density.device.index, C.c_void_p(density.data_ptr()), nz, ny, nx, _spacing(grid), _lib.f3(grid.origin),
        C.byref(mv.struct), C.byref(cv.struct), C.c_void_p(out.data_ptr()), _stream(density, stream))
    _lib.raise_for(rc)
    return out


PHOTON_DEPTH_MODES = {"march": 0, "lattice": 1}


def photon_depth_mode(gpu_id: int = 0, mode: str | None = None) -> str:
    """Select how photon calls on ``gpu_id`` compute the radiological depth
    ("march": the reference's per-voxel 1 mm march; "lattice": the default,
    the beam's-eye-view ray lattice with the march as its fallback) and
    return the mode in force."""
    lib = _lib.load()
    if mode is not None:
        if mode not in PHOTON_DEPTH_MODES:
            raise ValueError("photon depth mode must be one of %s" % sorted(PHOTON_DEPTH_MODES))
        _lib.raise_for(lib.dc_photon_set_depth_mode(gpu_id, PHOTON_DEPTH_MODES[mode]))
    cur = C.c_int(-1)
    _lib.raise_for(lib.dc_photon_get_depth_mode(gpu_id, C.byref(cur)))
    return {v: k for k, v in PHOTON_DEPTH_MODES.items()}[cur.value]


def photon_depth_marched(gpu_id: int = 0) -> int:
    """Voxels the last lattice depth pass on ``gpu_id`` marched exactly (-1:
    the last pass marched every voxel, or none ran).  Synchronises."""
    v = C.c_longlong(0)
    _lib.raise_for(_lib.load().dc_photon_depth_stats(gpu_id, C.byref(v)))
    return int(v.value)


def profile(gpu_id: int = 0, enable: bool | None = None, reset: bool = False):
    """Kernel timing control: enable/disable/reset, and read {kernel: (launches, ms)}."""
    lib = _lib.load()
    if enable is not None:
        _lib.raise_for(lib.dc_profile_enable(gpu_id, int(enable)))
    if reset:
        _lib.raise_for(lib.dc_profile_reset(gpu_id))
    return _lib.profile_read(gpu_id)


class ProtonBeamPlan:
    """One proton beam resident on a device, for plan optimisation.

    Holds the sorted spot and layer tables and the depth-dose tables on the
    GPU (C ABI ``dc_proton_beam_*``).  Given the beam's smoothed WET it gives
    the dose for any spot weights, the adjoint D^T g of a dose gradient, and the
    dose-influence matrix in CSR.  Spot-indexed tensors follow the order of
    ``beam.spot_list``."""

    def __init__(self, grid, beam, model, device="cuda", spots=None):
        dev = torch.device(device)
        if dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        sp = np.ascontiguousarray(beam.spot_list if spots is None else spots, dtype=np.float32).reshape(-1, 4)
        self.n_spots = sp.shape[0]
        dvp = np.ascontiguousarray(model.divergence_params, dtype=np.float32)
        ld, ls, li = (np.ascontiguousarray(a, dtype=np.float32) for a in (model.lut_depths, model.lut_sigmas,
                                                                          model.lut_idds))
        self._mu0 = torch.as_tensor(sp[:, 2].copy(), device=dev)
        self._grid, self._beam, self._model = grid, beam, model
        self._h = C.c_void_p()
        self._sp, self._dvp, self._luts = sp, dvp, (ld, ls, li)
        self._created_for = None

    def _handle(self, shape):
        if self._created_for == shape:
            return self._h
        self.close()
        lib = _lib.load()
        nz, ny, nx = shape
        ld, ls, li = self._luts
        h = C.c_void_p()
        with torch.cuda.device(self.device):
            rc = lib.dc_proton_beam_create(
                self.device.index, nz, ny, nx, _spacing(self._grid), _lib.f3(self._grid.origin),
                _lib.f3(self._beam.iso), float(self._beam.gantry_angle), float(self._beam.couch_angle),
                float(self._model.VSADX), float(self._model.VSADY), self._dvp.ctypes.data_as(C.c_void_p),
                ld.shape[0], self._dvp.shape[1], ld.ctypes.data_as(C.c_void_p), ls.ctypes.data_as(C.c_void_p),
                li.ctypes.data_as(C.c_void_p), ld.shape[1], self._sp.ctypes.data_as(C.c_void_p), self.n_spots,
                C.byref(h))
        _lib.raise_for(rc)
        self._h, self._created_for = h, shape
        return h

    def close(self):
        if self._h:
            _lib.load().dc_proton_beam_destroy(self._h)
            self._h = C.c_void_p()
            self._created_for = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def mu(self) -> torch.Tensor:
        """The MU column of the spot list, on the device."""
        return self._mu0

    def dose(self, wet: torch.Tensor, mu: torch.Tensor | None = None, out=None, stream=None) -> torch.Tensor:
        _check_volume(wet, "wet")
        h = self._handle(tuple(wet.shape))
        out = _out(wet, out)
        mu_p = None
        if mu is not None:
            mu = mu.detach().to(device=wet.device, dtype=torch.float32).contiguous()
            if mu.numel() != self.n_spots:
                raise ValueError("mu must hold one weight per spot")
            mu_p = C.c_void_p(mu.data_ptr())
        rc = _lib.load().dc_proton_beam_dose(h, C.c_void_p(wet.data_ptr()), mu_p, C.c_void_p(out.data_ptr()),
                                             _stream(wet, stream))
        _lib.raise_for(rc)
        return out

    def adjoint(self, wet: torch.Tensor, grad_dose: torch.Tensor, stream=None) -> torch.Tensor:
        """D^T g: float64 tensor with one entry per spot."""
        _check_volume(wet, "wet")
        g = grad_dose.detach().to(device=wet.device, dtype=torch.float32).contiguous()
        if g.shape != wet.shape:
            raise ValueError("grad_dose must have the volume's shape")
        h = self._handle(tuple(wet.shape))
        out = torch.empty(self.n_spots, dtype=torch.float64, device=wet.device)
        rc = _lib.load().dc_proton_beam_adjoint(h, C.c_void_p(wet.data_ptr()), C.c_void_p(g.data_ptr()),
                                                C.c_void_p(out.data_ptr()), _stream(wet, stream))
        _lib.raise_for(rc)
        return out

    @staticmethod
    def _voxels(voxels: torch.Tensor, device) -> torch.Tensor:
        v = voxels.to(device=device, dtype=torch.int32).reshape(-1).contiguous()
        if v.numel() >= 2 ** 31:
            raise ValueError("voxel lists are limited to 2^31 - 1 entries")
        return v

    def dose_list(self, wet: torch.Tensor, voxels: torch.Tensor, mu: torch.Tensor | None = None,
                  stream=None) -> torch.Tensor:
        """Dose (float32) at the listed voxels only (flat indices into the
        grid, best sorted); entries outside the grid give 0."""
        _check_volume(wet, "wet")
        h = self._handle(tuple(wet.shape))
        vox = self._voxels(voxels, wet.device)
        out = torch.empty(vox.numel(), dtype=torch.float32, device=wet.device)
        mu_p = None
        if mu is not None:
            mu = mu.detach().to(device=wet.device, dtype=torch.float32).contiguous()
            if mu.numel() != self.n_spots:
                raise ValueError("mu must hold one weight per spot")
            mu_p = C.c_void_p(mu.data_ptr())
        _lib.raise_for(_lib.load().dc_proton_beam_dose_list(h, C.c_void_p(wet.data_ptr()), mu_p,
                                                            C.c_void_p(vox.data_ptr()), vox.numel(),
                                                            C.c_void_p(out.data_ptr()), _stream(wet, stream)))
        return out

    def adjoint_list(self, wet: torch.Tensor, voxels: torch.Tensor, grad: torch.Tensor, stream=None) -> torch.Tensor:
        """D^T g for a gradient given at the listed voxels only (float64,
        one entry per spot)."""
        _check_volume(wet, "wet")
        h = self._handle(tuple(wet.shape))
        vox = self._voxels(voxels, wet.device)
        g = grad.detach().to(device=wet.device, dtype=torch.float32).reshape(-1).contiguous()
        if g.numel() != vox.numel():
            raise ValueError("one gradient value per listed voxel is required")
        out = torch.empty(self.n_spots, dtype=torch.float64, device=wet.device)
        _lib.raise_for(_lib.load().dc_proton_beam_adjoint_list(h, C.c_void_p(wet.data_ptr()),
                                                               C.c_void_p(vox.data_ptr()), vox.numel(),
                                                               C.c_void_p(g.data_ptr()), C.c_void_p(out.data_ptr()),
                                                               _stream(wet, stream)))
        return out

    def influence_csr(self, wet: torch.Tensor, cutoff: float = 1e-4, stream=None):
        """(row_ptr int64[n_voxels+1], col int32[nnz], val float32[nnz]) of the
        voxels x spots influence matrix, entries >= cutoff x the spot's maximum."""
        _check_volume(wet, "wet")
        h = self._handle(tuple(wet.shape))
        lib = _lib.load()
        nnz = C.c_longlong(0)
        _lib.raise_for(lib.dc_proton_beam_influence_nnz(h, C.c_void_p(wet.data_ptr()), float(cutoff),
                                                        C.byref(nnz), _stream(wet, stream)))
        n_vox = wet.numel()
        row_ptr = torch.empty(n_vox + 1, dtype=torch.int64, device=wet.device)
        col = torch.empty(max(nnz.value, 1), dtype=torch.int32, device=wet.device)
        val = torch.empty(max(nnz.value, 1), dtype=torch.float32, device=wet.device)
        _lib.raise_for(lib.dc_proton_beam_influence_csr(h, C.c_void_p(wet.data_ptr()), float(cutoff),
                                                        C.c_void_p(row_ptr.data_ptr()), C.c_void_p(col.data_ptr()),
                                                        C.c_void_p(val.data_ptr()), nnz.value, _stream(wet, stream)))
        return row_ptr, col[:nnz.value], val[:nnz.value]


class _ProtonDoseFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, mu, wet, plan):
        ctx.plan = plan
        ctx.save_for_backward(wet)
        ctx.mu_dtype = mu.dtype
        return plan.dose(wet, mu)

    @staticmethod
    def backward(ctx, grad_dose):
        (wet,) = ctx.saved_tensors
        g = ctx.plan.adjoint(wet, grad_dose)
        return g.to(ctx.mu_dtype), None, None


class _ProtonDoseListFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, mu, wet, plan, voxels):
        ctx.plan, ctx.voxels = plan, voxels
        ctx.save_for_backward(wet)
        ctx.mu_dtype = mu.dtype
        return plan.dose_list(wet, voxels, mu)

    @staticmethod
    def backward(ctx, grad):
        (wet,) = ctx.saved_tensors
        return ctx.plan.adjoint_list(wet, ctx.voxels, grad).to(ctx.mu_dtype), None, None, None


def proton_dose_list_autograd(mu: torch.Tensor, wet: torch.Tensor, plan: "ProtonBeamPlan",
                              voxels: torch.Tensor) -> torch.Tensor:
    """Differentiable dose of one beam at the listed voxels only (the voxel-
    list forms of the pencil-beam kernel and of its adjoint)."""
    return _ProtonDoseListFn.apply(mu, wet, plan, voxels)


def proton_dose_autograd(mu: torch.Tensor, wet: torch.Tensor, plan: ProtonBeamPlan) -> torch.Tensor:
    """Differentiable dose of one beam in its spot weights: forward is the
    pencil-beam kernel, backward the hand-written adjoint kernel (D^T g)."""
    return _ProtonDoseFn.apply(mu, wet, plan)


class ProtonBatch:
    """Many IMPT plans on one device, evaluated by one persistent launch.

    ``add_plan(grid, rlsp)`` takes a CT grid (spacing/origin, any anisotropic
    spacing) and its RLSP volume (CUDA tensor); ``add_beam(plan_id, beam)``
    takes an IMPTBeam-like object (iso, gantry_angle, couch_angle,
    spot_list).  After ``commit()``, ``wet()`` computes every beam's WET and
    ``dose(mu)`` every plan's dose (``self.doses[plan_id]``); both only enqueue
    device work, so they can be captured with ``torch.cuda.CUDAGraph``.
    ``autotune()`` times the kernel's tile shapes on this workload and keeps
    the fastest (cached in a JSON file keyed by the workload and GPU)."""

    def __init__(self, model, device="cuda"):
        dev = torch.device(device)
        if dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        self.model = model
        dvp = np.ascontiguousarray(model.divergence_params, dtype=np.float32)
        luts = [np.ascontiguousarray(a, dtype=np.float32) for a in (model.lut_depths, model.lut_sigmas,
                                                                    model.lut_idds)]
        h = C.c_void_p()
        with torch.cuda.device(dev):
            rc = _lib.load().dc_proton_batch_create(
                dev.index, dvp.ctypes.data_as(C.c_void_p), dvp.shape[0], dvp.shape[1],
                luts[0].ctypes.data_as(C.c_void_p), luts[1].ctypes.data_as(C.c_void_p),
                luts[2].ctypes.data_as(C.c_void_p), luts[0].shape[1], float(model.VSADX), float(model.VSADY),
                C.byref(h))
        _lib.raise_for(rc)
        self._h = h
        self.rlsp, self.doses, self.wets, self.beam_plan, self.beam_spots = [], [], [], [], []
        self.variant = 0
        self.committed = False

    def add_plan(self, grid, rlsp: torch.Tensor) -> int:
        _check_volume(rlsp, "rlsp")
        dose = torch.zeros_like(rlsp)
        pid = C.c_int()
        nz, ny, nx = rlsp.shape
        sp = np.asarray(grid.spacing, dtype=np.float32).reshape(-1)
        sp3 = (sp[0], sp[0], sp[0]) if sp.size == 1 else (sp[0], sp[1], sp[2])
        _lib.raise_for(_lib.load().dc_proton_batch_add_plan(self._h, nz, ny, nx, _lib.f3(sp3), _lib.f3(grid.origin),
                                                            C.c_void_p(rlsp.data_ptr()), C.c_void_p(dose.data_ptr()),
                                                            C.byref(pid)))
        self.rlsp.append(rlsp)
        self.doses.append(dose)
        return pid.value

    def add_beam(self, plan_id: int, beam) -> int:
        wet = torch.empty_like(self.rlsp[plan_id])
        sp = np.ascontiguousarray(beam.spot_list, dtype=np.float32).reshape(-1, 4)
        bid = C.c_int()
        _lib.raise_for(_lib.load().dc_proton_batch_add_beam(
            self._h, plan_id, _lib.f3(beam.iso), float(beam.gantry_angle), float(beam.couch_angle),
            sp.ctypes.data_as(C.c_void_p), sp.shape[0], C.c_void_p(wet.data_ptr()), C.byref(bid)))
        self.wets.append(wet)
        self.beam_plan.append(plan_id)
        self.beam_spots.append(sp)
        return bid.value

    def add_impt_plan(self, dose_grid, plan, rlsp: torch.Tensor | None = None) -> int:
        """Add a whole IMPTPlan (for instance one read by
        ``IMPTPlan.readPlanDicom``) on its IMPTDoseGrid: the grid's RLSP
        (``RLSPFromHU`` of the plan's machine unless given) and every beam.
        Beams are matched to beam models by range-shifter label as
        ``computeIMPTPlan`` does (plan_impt.py:124-160); all must use this
        batch's model.  The plan's dose is ``self.doses[pid]`` per fraction;
        ``plan_dose(pid)`` applies ``n_fractions`` as computeIMPTPlan does."""
        labels = list(np.asarray(plan.dicom_rangeshifter_label).astype(str))
        for beam in plan.beam_list:
            if str(beam.dicom_rangeshifter_label) not in labels:
                raise ValueError("Beam model not found for rangeshifter ID %s" % beam.dicom_rangeshifter_label)
            m = plan.beam_models[labels.index(str(beam.dicom_rangeshifter_label))]
            if not (np.array_equal(np.asarray(m.divergence_params), np.asarray(self.model.divergence_params)) and
                    np.array_equal(np.asarray(m.lut_idds), np.asarray(self.model.lut_idds))):
                raise ValueError("beam with range shifter %s needs another beam model than this batch's"
                                 % beam.dicom_rangeshifter_label)
        if rlsp is None:
            rlsp = torch.from_numpy(np.ascontiguousarray(dose_grid.RLSPFromHU(plan.machine_name),
                                                         dtype=np.float32)).to(self.device)
        pid = self.add_plan(dose_grid, rlsp)
        for beam in plan.beam_list:
            self.add_beam(pid, beam)
        if not hasattr(self, "n_fractions"):
            self.n_fractions = {}
        self.n_fractions[pid] = float(plan.n_fractions)
        return pid

    def plan_dose(self, pid: int) -> torch.Tensor:
        """Dose of plan ``pid`` over all fractions (the last ``dose()``)."""
        return self.doses[pid] * getattr(self, "n_fractions", {}).get(pid, 1.0)

    def commit(self):
        lib = _lib.load()
        _lib.raise_for(lib.dc_proton_batch_commit(self._h))
        n = [C.c_int() for _ in range(4)]
        _lib.raise_for(lib.dc_proton_batch_info(self._h, *[C.byref(x) for x in n]))
        self.n_plans, self.n_beams, self.n_spots, self.n_variants = (x.value for x in n)
        offs = []
        for b in range(self.n_beams):
            o = C.c_int()
            _lib.raise_for(lib.dc_proton_batch_beam_spot_offset(self._h, b, C.byref(o)))
            offs.append(o.value)
        self.spot_offsets = offs
        mu = np.zeros(self.n_spots, np.float32)
        for b, sp in enumerate(self.beam_spots):
            mu[offs[b]:offs[b] + sp.shape[0]] = sp[:, 2]
        self.mu0 = torch.as_tensor(mu, device=self.device)
        self.committed = True
        return self

    def wet(self, stream=None):
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        _lib.raise_for(_lib.load().dc_proton_batch_wet(self._h, C.c_void_p(s.cuda_stream)))

    def dose(self, mu: torch.Tensor | None = None, variant: int | None = None, stream=None):
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        mp = None
        if mu is not None:
            if mu.device != self.device or mu.dtype != torch.float32 or not mu.is_contiguous() or \
                    mu.numel() != self.n_spots:
                raise ValueError("mu must be a contiguous float32 tensor with one weight per spot on the batch's device")
            mp = C.c_void_p(mu.data_ptr())
        v = self.variant if variant is None else variant
        _lib.raise_for(_lib.load().dc_proton_batch_dose(self._h, mp, int(v), C.c_void_p(s.cuda_stream)))
        return self.doses

    def influence_csr(self, beam_id: int, cutoff: float = 1e-4, stream=None):
        """(row_ptr int64[n_voxels+1], col int32[nnz], val float32[nnz]) of
        beam ``beam_id``'s voxels x spots influence matrix on its plan's grid
        (after ``wet()``): entries >= cutoff x the spot's maximum, columns in
        the beam's spot-list order.  Count, then fill: the only allocations
        are the returned arrays."""
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        lib = _lib.load()
        n_vox = self.rlsp[self.beam_plan[beam_id]].numel()
        row_ptr = torch.empty(n_vox + 1, dtype=torch.int64, device=self.device)
        nnz = C.c_longlong(0)
        _lib.raise_for(lib.dc_proton_batch_influence_count(self._h, int(beam_id), float(cutoff),
                                                            C.c_void_p(row_ptr.data_ptr()), C.byref(nnz),
                                                            C.c_void_p(s.cuda_stream)))
        col = torch.empty(max(nnz.value, 1), dtype=torch.int32, device=self.device)
        val = torch.empty(max(nnz.value, 1), dtype=torch.float32, device=self.device)
        _lib.raise_for(lib.dc_proton_batch_influence_fill(self._h, int(beam_id), C.c_void_p(row_ptr.data_ptr()),
                                                           C.c_void_p(col.data_ptr()), C.c_void_p(val.data_ptr()),
                                                           col.numel(), C.c_void_p(s.cuda_stream)))
        return row_ptr, col[:nnz.value], val[:nnz.value]

    def autotune(self, cache_path: str | None = None, repeats: int = 3) -> int:
        """Time every tile shape of the batch dose kernel on this workload and
        keep the fastest; results are cached in ``cache_path`` (JSON)."""
        import json
        import os
        key = "%s|%d plans|%d beams|%d spots|%s" % (
            torch.cuda.get_device_name(self.device), self.n_plans, self.n_beams, self.n_spots,
            ";".join("x".join(str(d) for d in r.shape) for r in self.rlsp))
        cache = {}
        if cache_path and os.path.exists(cache_path):
            with open(cache_path) as f:
                cache = json.load(f)
        if key in cache:
            self.variant = int(cache[key]["variant"])
            return self.variant
        times = []
        for v in range(self.n_variants):
            self.dose(variant=v)
            torch.cuda.synchronize(self.device)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(repeats):
                self.dose(variant=v)
            b.record()
            torch.cuda.synchronize(self.device)
            times.append(a.elapsed_time(b) / repeats)
        self.variant = int(np.argmin(times))
        if cache_path:
            cache[key] = {"variant": self.variant, "ms": times}
            with open(cache_path, "w") as f:
                json.dump(cache, f, indent=1)
        self.tune_ms = times
        return self.variant

    def close(self):
        if self._h:
            _lib.load().dc_proton_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PhotonBeam:
    """A photon calculation kept on one device for a fixed grid (C ABI
    ``dc_photon_beam_*``): one ray trace + TERMA pass per control point, after
    which the full CCCS dose and the CCCS dose at any list of voxels (a sparse
    probe) come from the same TERMA.  Results equal ``photon_dose``."""

    def __init__(self, grid, shape, device="cuda"):
        dev = torch.device(device)
        if dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        self.shape = tuple(int(s) for s in shape)
        self.spacing = np.asarray(grid.spacing, np.float32).reshape(-1)
        if self.spacing.size == 1:
            self.spacing = np.repeat(self.spacing, 3)
        self._grid = grid
        self._h = C.c_void_p()
        nz, ny, nx = self.shape
        with torch.cuda.device(dev):
            _lib.raise_for(_lib.load().dc_photon_beam_create(dev.index, nz, ny, nx, _spacing(grid),
                                                              _lib.f3(grid.origin), C.byref(self._h)))
        self.n_probe = 0
        self._views = None

    def close(self):
        if self._h:
            _lib.load().dc_photon_beam_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _s(self, stream):
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        return C.c_void_p(s.cuda_stream)

    def set_density(self, density: torch.Tensor, stream=None):
        _check_volume(density, "density")
        if tuple(density.shape) != self.shape:
            raise ValueError("'density' must have the beam's shape %s." % (self.shape,))
        _lib.raise_for(_lib.load().dc_photon_beam_set_density(self._h, C.c_void_p(density.data_ptr()),
                                                               self._s(stream)))

    def terma(self, model, cp, out=None, views=None, stream=None) -> torch.Tensor | None:
        """Ray trace + TERMA of control point ``cp``; returns the TERMA volume
        when ``out`` is given (or ``out=True`` to allocate it)."""
        mv, cv = views if views is not None else (PhotonModelView(model), ControlPointView(cp))
        self._views = (mv, cv)  # keep the packed arrays alive while the call is in flight
        if out is True:
            out = torch.empty(self.shape, dtype=torch.float32, device=self.device)
        ptr = C.c_void_p(out.data_ptr()) if out is not None else None
        _lib.raise_for(_lib.load().dc_photon_beam_terma(self._h, C.byref(mv.struct), C.byref(cv.struct), ptr,
                                                         self._s(stream)))
        self.n_probe = self.probe_voxels(host=False)[1]
        return out

    def probe_config(self, lattice_stride: int):
        """Probe lattice stride (0: cone lines and profiles only)."""
        _lib.raise_for(_lib.load().dc_photon_beam_probe_config(self._h, int(lattice_stride)))

    def dose(self, out=None, stream=None) -> torch.Tensor:
        if out is None:
            out = torch.empty(self.shape, dtype=torch.float32, device=self.device)
        _lib.raise_for(_lib.load().dc_photon_beam_dose(self._h, C.c_void_p(out.data_ptr()), self._s(stream)))
        return out

    def dose_sweep(self, out=None, stream=None) -> torch.Tensor:
        """The CCCS by cone-direction sweeps over line lattices: an
        approximation of ``dose`` (no per-voxel kernel tilt, windows
        interpolated between lattice lines); synchronises once."""
        if out is None:
            out = torch.empty(self.shape, dtype=torch.float32, device=self.device)
        _lib.raise_for(_lib.load().dc_photon_beam_dose_sweep(self._h, C.c_void_p(out.data_ptr()), self._s(stream)))
        return out

    def select_probe(self, stream=None) -> int:
        n = C.c_int()
        _lib.raise_for(_lib.load().dc_photon_beam_probe_select(self._h, C.byref(n), self._s(stream)))
        self.n_probe = n.value
        return self.n_probe

    def probe_voxels(self, host: bool = True) -> tuple[int, int, np.ndarray | None]:
        """(device pointer, count, host copy or None) of the selected probe
        voxels (selected by ``terma``)."""
        p, n = C.c_void_p(), C.c_int()
        lib = _lib.load()
        _lib.raise_for(lib.dc_photon_beam_probe_list(self._h, C.byref(p), C.byref(n), None, 0))
        if not host:
            return p.value or 0, n.value, None
        arr = np.empty(max(n.value, 1), np.int32)
        _lib.raise_for(lib.dc_photon_beam_probe_list(self._h, C.byref(p), C.byref(n), arr.ctypes.data_as(C.c_void_p),
                                                     arr.size))
        return p.value or 0, n.value, arr[:n.value]

    def probe(self, voxels: torch.Tensor | None = None, out=None, stream=None) -> torch.Tensor:
        """CCCS dose at ``voxels`` (int32 flat indices) or at the selected probe."""
        n = int(voxels.numel()) if voxels is not None else self.n_probe
        if out is None:
            out = torch.empty(max(n, 1), dtype=torch.float32, device=self.device)[:n]
        vp = C.c_void_p(voxels.data_ptr()) if voxels is not None else None
        _lib.raise_for(_lib.load().dc_photon_beam_probe(self._h, vp, n, C.c_void_p(out.data_ptr()),
                                                         self._s(stream)))
        return out


class PhotonFluenceBeam:
    """One photon control point on the device with a beamlet fluence map:
    the dose as a linear function of the map and its adjoint (C ABI
    ``dc_photon_beam_fluence_dose`` / ``_adjoint``).

    The map is a grid of beamlets on the beam's-eye-view isocentre plane
    (head frame, mm): beamlet (ia, ib) sits at (a0 + ia*pitch, b0 + ib*pitch)
    and values are a float32 tensor of shape (nb, na).  Each voxel's TERMA and
    electron term are scaled by the map's bilinear interpolation at the
    voxel's ray, so ``dose(ones)`` is the control point's CCCS dose (bit for
    bit) and ``dose`` is linear in the map; ``adjoint(g)`` is the exact
    gradient d(sum g D)/d map in float64 through the transpose of the
    collapsed-cone superposition.  ``photon_fluence_dose_autograd`` wraps both
    in a torch.autograd.Function.  ``field_map`` builds a map covering the
    control point's open MLC field."""

    def __init__(self, density: torch.Tensor, grid, model, cp, na: int, nb: int, a0: float, b0: float,
                 pitch: float, views=None):
        self.beam = PhotonBeam(grid, density.shape, device=density.device)
        self.beam.set_density(density)
        self.beam.terma(model, cp, views=views)
        self.device = density.device
        self.shape = tuple(density.shape)
        self.map = _lib.FluenceMap(int(na), int(nb), float(a0), float(b0), float(pitch))
        self.na, self.nb = int(na), int(nb)

    @classmethod
    def field_map(cls, density, grid, model, cp, pitch: float = 5.0, margin: float = 10.0, views=None):
        """A map of ``pitch`` mm beamlets over the control point's open MLC
        field (leaf pairs with x2 > x1, projected to the isocentre plane by the
        leaves' own coordinates) plus ``margin`` mm on every side."""
        mlc = np.asarray(cp.mlc, np.float32)
        openp = mlc[:, 1] > mlc[:, 0]
        if not openp.any():
            raise ValueError("the control point has no open leaf pair")
        a_lo, a_hi = float(mlc[openp, 0].min()) - margin, float(mlc[openp, 1].max()) + margin
        yb = mlc[openp, 2] - 0.5 * mlc[openp, 3]
        yt = mlc[openp, 2] + 0.5 * mlc[openp, 3]
        b_lo, b_hi = float(yb.min()) - margin, float(yt.max()) + margin
        na = int(np.ceil((a_hi - a_lo) / pitch)) + 1
        nb = int(np.ceil((b_hi - b_lo) / pitch)) + 1
        return cls(density, grid, model, cp, na, nb, a_lo, b_lo, pitch, views=views)

    def _check_map(self, t: torch.Tensor, dtype):
        if tuple(t.shape) != (self.nb, self.na) or t.dtype != dtype or t.device != self.device or \
                not t.is_contiguous():
            raise ValueError("fluence must be a contiguous %s tensor of shape (%d, %d) on %s"
                             % (dtype, self.nb, self.na, self.device))

    def dose(self, fluence: torch.Tensor, out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
        f = fluence.detach().to(device=self.device, dtype=torch.float32).contiguous()
        self._check_map(f, torch.float32)
        out = torch.empty(self.shape, dtype=torch.float32, device=self.device) if out is None else out
        _check_volume(out, "out")
        _lib.raise_for(_lib.load().dc_photon_beam_fluence_dose(self.beam._h, C.byref(self.map),
                                                                C.c_void_p(f.data_ptr()), C.c_void_p(out.data_ptr()),
                                                                self.beam._s(stream)))
        return out

    def adjoint(self, grad_dose: torch.Tensor, stream=None) -> torch.Tensor:
        g = grad_dose.detach().to(device=self.device, dtype=torch.float32).contiguous()
        if tuple(g.shape) != self.shape:
            raise ValueError("grad_dose must have the volume's shape")
        out = torch.empty((self.nb, self.na), dtype=torch.float64, device=self.device)
        _lib.raise_for(_lib.load().dc_photon_beam_fluence_adjoint(self.beam._h, C.byref(self.map),
                                                                   C.c_void_p(g.data_ptr()),
                                                                   C.c_void_p(out.data_ptr()), self.beam._s(stream)))
        return out

    def close(self):
        self.beam.close()


class _PhotonFluenceFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, fluence, beam):
        ctx.beam = beam
        return beam.dose(fluence)

    @staticmethod
    def backward(ctx, grad):
        return ctx.beam.adjoint(grad).to(torch.float32), None


def photon_fluence_dose_autograd(fluence: torch.Tensor, beam: PhotonFluenceBeam) -> torch.Tensor:
    """Differentiable photon dose in the beamlet fluence map: forward is the
    modulated TERMA + CCCS, backward the hand-written CCCS transpose."""
    return _PhotonFluenceFn.apply(fluence, beam)


def gamma_counts(eval_dose: torch.Tensor, spacing, ref: torch.Tensor, voxels: torch.Tensor | int | None = None,
                 n: int | None = None, dose_norm: float = 0.0, dta_mm: float = 2.0, dd_frac: float = 0.02,
                 cutoff_frac: float = 0.1, counts: torch.Tensor | None = None, stream=None) -> torch.Tensor:
    """Gamma index of ``eval_dose`` against reference doses on the device
    (C ABI ``dc_gamma``): ``ref`` is a volume (``voxels`` None) or the doses at
    the listed voxels (a tensor of int32 indices, or a raw device pointer with
    ``n``).  Returns the int32 device tensor [evaluated, passed, -, -]."""
    _check_volume(eval_dose, "eval_dose")
    nz, ny, nx = eval_dose.shape
    if counts is None:
        counts = torch.empty(4, dtype=torch.int32, device=eval_dose.device)
    sp = np.asarray(spacing, np.float32).reshape(-1)
    sp3 = _lib.f3(sp if sp.size == 3 else np.repeat(sp, 3))
    if voxels is None:
        vp, count = None, nz * ny * nx
    elif isinstance(voxels, torch.Tensor):
        vp, count = C.c_void_p(voxels.data_ptr()), int(voxels.numel())
    else:
        vp, count = C.c_void_p(int(voxels)), int(n)
    _lib.raise_for(_lib.load().dc_gamma(
        eval_dose.device.index, C.c_void_p(eval_dose.data_ptr()), nz, ny, nx, sp3, vp,
        C.c_void_p(ref.data_ptr()), count, float(dose_norm), float(dta_mm), float(dd_frac), float(cutoff_frac),
        C.c_void_p(counts.data_ptr()), _stream(eval_dose, stream)))
    return counts


def _table(t):
    th, tv = (np.ascontiguousarray(np.asarray(a, np.float64)) for a in t)
    if th.ndim != 1 or th.shape != tv.shape:
        raise ValueError("an HU table is two 1-D arrays of the same length")
    return th, tv


def hu_convert(hu: torch.Tensor, table, out=None, stream=None) -> torch.Tensor:
    """HU -> table value (relative stopping power or density) on the device;
    equals np.interp(hu, *table).astype(float32) bit for bit."""
    _check_volume(hu, "hu")
    out = _out(hu, out)
    th, tv = _table(table)
    nz, ny, nx = hu.shape
    _lib.raise_for(_lib.load().dc_hu_convert_dev(
        hu.device.index, C.c_void_p(hu.data_ptr()), nz, ny, nx, th.ctypes.data_as(C.c_void_p),
        tv.ctypes.data_as(C.c_void_p), th.size, C.c_void_p(out.data_ptr()), _stream(hu, stream)))
    return out


def proton_wet_hu(hu: torch.Tensor, grid, beam, model, table, out=None, stream=None) -> torch.Tensor:
    """``proton_wet`` from an HU volume: the HU -> RLSP conversion writes the
    ray tracer's texture directly (no RLSP volume in between)."""
    _check_volume(hu, "hu")
    out = _out(hu, out)
    th, tv = _table(table)
    nz, ny, nx = hu.shape
    _lib.raise_for(_lib.load().dc_proton_raytrace_hu_dev(
        hu.device.index, C.c_void_p(hu.data_ptr()), nz, ny, nx, _spacing(grid), _lib.f3(grid.origin),
        th.ctypes.data_as(C.c_void_p), tv.ctypes.data_as(C.c_void_p), th.size, _lib.f3(beam.iso),
        float(beam.gantry_angle), float(beam.couch_angle), float(model.VSADX), float(model.VSADY),
        C.c_void_p(out.data_ptr()), _stream(hu, stream)))
    return out


def photon_plan_dose(volume: torch.Tensor, grid, model, cps, weights, out: torch.Tensor, hu_table=None, views=None,
                     stream=None) -> torch.Tensor:
    """out += sum_i weights[i] * CCCS dose of control point cps[i], in one call
    (the volume is loaded once; with ``hu_table`` it is an HU volume converted
    on the device).  weights are float64 (output factors)."""
    _check_volume(volume, "volume")
    _check_volume(out, "out")
    mv = views if views is not None else PhotonModelView(model)
    cvs = [ControlPointView(cp) for cp in cps]
    arr = (_lib.ControlPoint * max(len(cvs), 1))(*[c.struct for c in cvs])
    w = np.ascontiguousarray(np.asarray(weights, np.float64).reshape(-1))
    if w.size != len(cvs):
        raise ValueError("one weight per control point is required")
    if hu_table is not None:
        th, tv = _table(hu_table)
        tp = (th.ctypes.data_as(C.c_void_p), tv.ctypes.data_as(C.c_void_p), th.size)
    else:
        tp = (None, None, 0)
    nz, ny, nx = volume.shape
    _lib.raise_for(_lib.load().dc_photon_plan_dose_dev(
        volume.device.index, C.c_void_p(volume.data_ptr()), int(hu_table is not None), tp[0], tp[1], tp[2], nz, ny,
        nx, _spacing(grid), _lib.f3(grid.origin), C.byref(mv.struct), C.cast(arr, C.c_void_p), len(cvs),
        w.ctypes.data_as(C.c_void_p), C.c_void_p(out.data_ptr()), _stream(volume, stream)))
    return out


class PhotonPlanBasis:
    """The control points of one photon beam as a linear dose basis on the
    device, for segment-weight (fluence) optimisation.

    ``basis[b]`` is the CCCS dose of control point b (``photon_dose`` of
    ``cps[b]``, before its output factor); the beam's dose for segment
    weights w is  D(w) = sum_b w_b OF_b basis[b]  (``dose``), with the
    reference plan loop's float32 += float32 * float64 arithmetic, so w = 1
    gives the plan loop's beam dose bit for bit.  ``adjoint(g)`` is the exact
    gradient  d(sum_v g_v D_v)/dw_b = OF_b sum_v g_v basis[b][v]  in float64
    (hand-written kernels ``dc_basis_combine_dev`` / ``dc_basis_adjoint_dev``).
    Gradients with respect to leaf positions or beamlet fluence would need
    the transpose of the collapsed-cone superposition and are not provided.
    """

    def __init__(self, density: torch.Tensor, grid, model, cps, output_factors=None, views=None):
        _check_volume(density, "density")
        self.device = density.device
        self.shape = tuple(density.shape)
        self.n = len(cps)
        if self.n < 1:
            raise ValueError("at least one control point is required")
        of = [float(model.outputFactor(cp)) for cp in cps] if output_factors is None else list(output_factors)
        if len(of) != self.n:
            raise ValueError("one output factor per control point is required")
        self.output_factors = torch.tensor(of, dtype=torch.float64, device=self.device)
        self.basis = torch.empty((self.n,) + self.shape, dtype=torch.float32, device=self.device)
        mv = views if views is not None else PhotonModelView(model)
        beam = PhotonBeam(grid, self.shape, device=self.device)
        try:
            beam.set_density(density)
            for b, cp in enumerate(cps):
                beam.terma(model, cp, views=(mv, ControlPointView(cp)))
                beam.dose(out=self.basis[b])
        finally:
            beam.close()

    def dose(self, weights: torch.Tensor | None = None, out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
        """Beam dose (float32 volume) for segment weights (default all 1)."""
        coef = self.output_factors if weights is None else \
            weights.detach().to(device=self.device, dtype=torch.float64).reshape(-1) * self.output_factors
        if coef.numel() != self.n:
            raise ValueError("one weight per control point is required")
        coef = coef.contiguous()
        out = torch.zeros(self.shape, dtype=torch.float32, device=self.device) if out is None else out.zero_()
        _check_volume(out, "out")
        _lib.raise_for(_lib.load().dc_basis_combine_dev(
            self.device.index, C.c_void_p(self.basis.data_ptr()), self.n, out.numel(), C.c_void_p(coef.data_ptr()),
            C.c_void_p(out.data_ptr()), _stream(out, stream)))
        return out

    def adjoint(self, grad_dose: torch.Tensor, stream=None) -> torch.Tensor:
        """Gradient with respect to the segment weights (float64, one per
        control point) of sum_v grad_dose_v D_v."""
        g = grad_dose.detach().to(device=self.device, dtype=torch.float32).contiguous()
        if tuple(g.shape) != self.shape:
            raise ValueError("grad_dose must have the volume's shape")
        out = torch.empty(self.n, dtype=torch.float64, device=self.device)
        _lib.raise_for(_lib.load().dc_basis_adjoint_dev(
            self.device.index, C.c_void_p(self.basis.data_ptr()), self.n, g.numel(), C.c_void_p(g.data_ptr()),
            C.c_void_p(out.data_ptr()), _stream(g, stream)))
        return out * self.output_factors


class _PhotonBasisFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, weights, basis):
        ctx.basis = basis
        ctx.w_dtype = weights.dtype
        return basis.dose(weights)

    @staticmethod
    def backward(ctx, grad_dose):
        return ctx.basis.adjoint(grad_dose).to(ctx.w_dtype), None


def photon_dose_autograd(weights: torch.Tensor, basis: PhotonPlanBasis) -> torch.Tensor:
    """Differentiable beam dose in the segment weights of a photon beam:
    forward is the basis combination, backward the adjoint kernel."""
    return _PhotonBasisFn.apply(weights, basis)
