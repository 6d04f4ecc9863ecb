"""IMRT plan API (mirror of DoseCUDA/plan_imrt.py).

Same classes, attributes and array layouts as the reference: in particular
``IMRTPhotonEnergy.kernel`` is the Fortran-ordered float32 (6, 6) array that
pandas produces and ``IMRTControlPoint.mlc`` is the (n_pairs, 4) transposed
view of a (4, n_pairs) array, which is how the reference's extension reads
them (dosemodule.cu:228-240, IMRTClasses.cu:292-297).  The dose calls go to
the sm_100a engine via ``dosecuda_b200.dose_kernels``.
"""
from __future__ import annotations

import os

import numpy as np
import pandas as pd

from . import dose_kernels
from .lookup import read_key_values, table_path
from .plan import Beam, DoseGrid, Plan, VolumeObject, _pydicom


class IMRTPhotonEnergy:
    """Photon beam model of one nominal energy (reference plan_imrt.py:13-92)."""

    _REQUIRED = (
        "output_factor_equivalent_squares", "output_factor_values", "mu_calibration",
        "primary_source_distance", "scatter_source_distance", "mlc_distance",
        "scatter_source_weight", "electron_attenuation", "primary_source_size",
        "scatter_source_size", "profile_radius", "profile_intensities",
        "profile_softening", "spectrum_attenuation_coefficients", "spectrum_primary_weights",
        "spectrum_scatter_weights", "electron_source_weight", "has_xjaws", "has_yjaws",
        "electron_fitted_dmax", "jaw_transmission", "mlc_transmission",
    )

    def __init__(self, dicom_energy_label):
        self.dicom_energy_label = dicom_energy_label
        for name in self._REQUIRED:
            setattr(self, name, None)
        self.mlc_index = None
        self.mlc_widths = None
        self.mlc_offsets = None
        self.n_mlc_pairs = None
        self.kernel = None

    def validate_parameters(self):
        for name in self._REQUIRED:
            if getattr(self, name) is None:
                raise Exception(f"{name} not set in beam model")

    def outputFactor(self, cp):
        """Output factor from the MLC aperture's equivalent square (4 A / P over
        the open leaf pairs) by linear interpolation (reference plan_imrt.py:61-92)."""
        min_y, max_y, max_x_diff, area = 10000.0, -10000.0, 0.0, 0.0
        for i in range(cp.mlc.shape[0]):
            x1, x2, y_offset, y_width = cp.mlc[i, 0], cp.mlc[i, 1], cp.mlc[i, 2], cp.mlc[i, 3]
            area += (x2 - x1) * y_width
            opening = x2 - x1
            if opening > 3.0 and opening > max_x_diff:
                max_x_diff = opening
            if opening > 3.0:
                if (y_offset - y_width / 2.0) < min_y:
                    min_y = y_offset - y_width / 2.0
                if (y_offset + y_width / 2.0) > max_y:
                    max_y = y_offset + y_width / 2.0
        perimeter = 2 * (max_y - min_y) + 2 * max_x_diff
        equivalent_square = 4 * area / perimeter
        return np.interp(equivalent_square, self.output_factor_equivalent_squares, self.output_factor_values)


class IMRTControlPoint:
    def __init__(self, iso, mu, mlc, ga, ca, ta, xjaws, yjaws):
        self.iso = iso
        self.mu = mu
        self.mlc = mlc
        self.ga = ga
        self.ca = ca
        self.ta = ta
        self.xjaws = xjaws
        self.yjaws = yjaws


class IMRTDoseGrid(DoseGrid):
    def __init__(self):
        super().__init__()
        self.Density = []

    def DensityFromHU(self, machine_name):
        """Piecewise-linear HU -> relative electron density (reference plan_imrt.py:114-124)."""
        df = pd.read_csv(table_path("photons", machine_name, "HU_Density.csv"))
        return np.array(np.interp(self.HU, df["HU"].to_numpy(), df["Density"].to_numpy()), dtype=np.single)

    def computeIMRTPlan(self, plan, gpu_id=0, device=False):
        """Sum over beams and control points of output factor x CCCS dose, times
        the number of fractions (reference plan_imrt.py:126-158).

        ``device=True`` keeps the plan on the GPU: the HU volume is uploaded
        once and converted there; each beam's control points run in one call
        that accumulates output factor x dose on the device; the results are
        copied back once.  Same arithmetic as the host loop."""
        if device:
            return self._computeIMRTPlanDevice(plan, gpu_id)
        self.beam_doses = []
        self.dose = np.zeros(self.size, dtype=np.single)
        self.Density = self.DensityFromHU(plan.machine_name)
        if self.spacing[0] != self.spacing[1] or self.spacing[0] != self.spacing[2]:
            raise Exception("Spacing must be isotropic for IMPT dose calculation - consider resampling CT")
        vol = VolumeObject()
        vol.voxel_data = np.array(self.Density, dtype=np.single)
        vol.origin = np.array(self.origin, dtype=np.single)
        vol.spacing = np.array(self.spacing, dtype=np.single)
        labels = list(plan.dicom_energy_label.astype(str))
        for beam in plan.beam_list:
            if str(beam.dicom_energy_label) not in labels:
                raise ValueError("Beam model not found for beam energy %s" % beam.dicom_energy_label)
            model = plan.beam_models[labels.index(str(beam.dicom_energy_label))]
            beam_dose = np.zeros(self.Density.shape, dtype=np.single)
            for cp in beam.cp_list:
                of = model.outputFactor(cp)
                beam_dose += dose_kernels.photon_dose_cuda(model, vol, cp, gpu_id) * of
            self.beam_doses.append(beam_dose)
            self.dose += beam_dose
        self.dose *= plan.n_fractions


    def _computeIMRTPlanDevice(self, plan, gpu_id):
        import torch

        from . import engine
        from .dose_kernels import PhotonModelView
        if self.spacing[0] != self.spacing[1] or self.spacing[0] != self.spacing[2]:
            raise Exception("Spacing must be isotropic for IMPT dose calculation - consider resampling CT")
        dev = torch.device("cuda", gpu_id)
        df = pd.read_csv(table_path("photons", plan.machine_name, "HU_Density.csv"))
        table = (df["HU"].to_numpy(), df["Density"].to_numpy())
        hu = torch.as_tensor(np.ascontiguousarray(self.HU, dtype=np.single), device=dev)
        labels = list(plan.dicom_energy_label.astype(str))
        total = torch.zeros(hu.shape, dtype=torch.float32, device=dev)
        doses = []
        for beam in plan.beam_list:
            if str(beam.dicom_energy_label) not in labels:
                raise ValueError("Beam model not found for beam energy %s" % beam.dicom_energy_label)
            model = plan.beam_models[labels.index(str(beam.dicom_energy_label))]
            beam_dose = torch.zeros(hu.shape, dtype=torch.float32, device=dev)
            weights = [float(model.outputFactor(cp)) for cp in beam.cp_list]
            engine.photon_plan_dose(hu, self, model, beam.cp_list, weights, beam_dose, hu_table=table,
                                    views=PhotonModelView(model))
            doses.append(beam_dose)
            total += beam_dose
        total *= plan.n_fractions
        self.Density = engine.hu_convert(hu, table).cpu().numpy()
        self.beam_doses = [d.cpu().numpy() for d in doses]
        self.dose = total.cpu().numpy()


class IMRTBeam(Beam):
    def __init__(self):
        super().__init__()
        self.cp_list = []
        self.n_cps = 0
        self.dicom_energy_label = None

    def addControlPoint(self, cp):
        self.cp_list.append(cp)
        self.n_cps += 1


def _mlc_array(x12: np.ndarray, offsets: np.ndarray, widths: np.ndarray) -> np.ndarray:
    """(n_pairs, 4) = x1, x2, y_offset, y_width as the transpose of a
    (4, n_pairs) C array (the reference's layout, plan_imrt.py:371-372)."""
    stacked = np.array(np.vstack((x12, offsets.reshape(1, -1), widths.reshape(1, -1))), dtype=np.single)
    return np.transpose(stacked)


class IMRTPlan(Plan):
    def __init__(self, machine_name="VarianTrueBeamHF"):
        super().__init__()
        self.machine_name = machine_name
        el = pd.read_csv(table_path("photons", machine_name, "energy_labels.csv"))
        self.dicom_energy_label = el["dicom_energy_label"]
        self.folder_energy_label = el["folder_energy_label"]
        self.beam_models = []
        for d, f in zip(self.dicom_energy_label, self.folder_energy_label):
            bm = IMRTPhotonEnergy(d)
            self._load_beam_model_parameters(bm, machine_name, f)
            self.beam_models.append(bm)

    def _load_beam_model_parameters(self, beam_model, machine_name, folder_energy_label):
        base = table_path("photons", machine_name)
        mlc = pd.read_csv(os.path.join(base, "mlc_geometry.csv"))
        beam_model.mlc_index = mlc["mlc_pair_index"].to_numpy()
        beam_model.mlc_widths = mlc["width"].to_numpy()
        beam_model.mlc_offsets = mlc["center_offset"].to_numpy()
        beam_model.n_mlc_pairs = len(beam_model.mlc_index)
        kernel = pd.read_csv(os.path.join(base, folder_energy_label, "kernel.csv"))
        beam_model.kernel = np.array(kernel.to_numpy(), dtype=np.single)  # Fortran order, as the reference
        self._load_machine_geometry(beam_model, os.path.join(base, "machine_geometry.csv"))
        self._load_beam_parameters(beam_model, os.path.join(base, folder_energy_label, "beam_parameters.csv"))
        beam_model.validate_parameters()

    def _load_machine_geometry(self, beam_model, path):
        kv = read_key_values(path)
        for key in ("primary_source_distance", "scatter_source_distance", "mlc_distance"):
            if key in kv:
                setattr(beam_model, key, float(kv[key][0]))
        for key in ("has_xjaws", "has_yjaws"):
            if key in kv:
                setattr(beam_model, key, bool(kv[key][0]))

    _ARRAY_KEYS = ("output_factor_equivalent_squares", "output_factor_values", "profile_radius",
                   "profile_intensities", "profile_softening", "spectrum_attenuation_coefficients",
                   "spectrum_primary_weights", "spectrum_scatter_weights")
    _SCALAR_KEYS = ("mu_calibration", "scatter_source_weight", "electron_attenuation", "primary_source_size",
                    "scatter_source_size", "electron_source_weight", "electron_fitted_dmax", "jaw_transmission",
                    "mlc_transmission")

    def _load_beam_parameters(self, beam_model, path):
        kv = read_key_values(path)
        for key in self._ARRAY_KEYS:
            if key in kv:
                setattr(beam_model, key, np.array(kv[key], dtype=np.single))
        for key in self._SCALAR_KEYS:
            if key in kv:
                setattr(beam_model, key, float(kv[key][0]))

    def addSquareField(self, dicom_energy_label="6", dimx=10, dimy=10, mu=100, gantry_angle=0.0,
                       collimator_angle=0.0, table_angle=0.0):
        """One open dimx x dimy cm field shaped by the MLC (reference plan_imrt.py:353-382)."""
        model = self.beam_models[0]
        beam = IMRTBeam()
        beam.dicom_energy_label = dicom_energy_label
        iso = np.array([0.0, 0.0, 0.0], dtype=np.single)
        dimx *= 10.0
        dimy *= 10.0
        x12 = np.zeros((2, model.n_mlc_pairs), dtype=np.single)
        x12[0, :] = -dimx / 2.0
        x12[1, :] = dimx / 2.0
        outside = (model.mlc_offsets < -(dimy / 2.0)) | (model.mlc_offsets > (dimy / 2.0))
        x12[:, outside] = 0.0
        mlc = _mlc_array(x12, model.mlc_offsets, model.mlc_widths)
        jawx = np.array([-dimx / 2.0, dimx / 2.0], dtype=np.single)
        jawy = np.array([-dimy / 2.0, dimy / 2.0], dtype=np.single)
        beam.addControlPoint(IMRTControlPoint(iso, mu, mlc, gantry_angle, collimator_angle, table_angle, jawx, jawy))
        self.addBeam(beam)

    def readPlanDicom(self, plan_path):
        """Control points of an RT Plan (reference plan_imrt.py:273-351)."""
        pyd = _pydicom()
        ds = pyd.dcmread(plan_path)
        total_mu = ds.FractionGroupSequence[0].ReferencedBeamSequence[0].BeamMeterset
        self.n_fractions = float(ds.FractionGroupSequence[0].NumberOfFractionsPlanned)
        self.beam_list = []
        self.n_beams = 0
        model = self.beam_models[0]
        n_pairs = model.n_mlc_pairs

        def read_devices(cp):
            xj = yj = ml = None
            for ps in cp.BeamLimitingDevicePositionSequence:
                if ps.RTBeamLimitingDeviceType == "X":
                    xj = np.array(cp.BeamLimitingDevicePositionSequence[1].LeafJawPositions, dtype=np.single)
                if ps.RTBeamLimitingDeviceType == "Y":
                    yj = np.array(cp.BeamLimitingDevicePositionSequence[1].LeafJawPositions, dtype=np.single)
                if ps.RTBeamLimitingDeviceType == "MLCX":
                    ml = np.array(cp.BeamLimitingDevicePositionSequence[2].LeafJawPositions, dtype=np.single)
            return xj, yj, ml

        for b in ds.BeamSequence:
            if b.TreatmentDeliveryType != "TREATMENT":
                continue
            beam = IMRTBeam()
            cumulative_mu = 0.0
            ga = ca = ta = None
            xjaws = yjaws = mlc = None
            for cp in b.ControlPointSequence:
                if cp.ControlPointIndex == 0:
                    beam.dicom_energy_label = cp.NominalBeamEnergy
                    beam.iso = np.array([cp.IsocenterPosition[0], cp.IsocenterPosition[1], cp.IsocenterPosition[2]],
                                        dtype=np.single)
                    ca, ta, ga = cp.BeamLimitingDeviceAngle, cp.PatientSupportAngle, cp.GantryAngle
                    xjaws, yjaws, mlc = read_devices(cp)
                    continue
                mu = cp.CumulativeMetersetWeight - cumulative_mu
                if mlc is not None:
                    m = _mlc_array(np.reshape(mlc, (2, n_pairs)), model.mlc_offsets, model.mlc_widths)
                else:
                    x12 = np.zeros((2, n_pairs), dtype=np.single)
                    if xjaws is not None:
                        x12[0, :] = xjaws[0]
                        x12[1, :] = xjaws[1]
                    if yjaws is not None:
                        outside = (model.mlc_offsets < yjaws[0]) | (model.mlc_offsets > yjaws[1])
                        x12[:, outside] = 0.0
                    m = _mlc_array(x12, model.mlc_offsets, model.mlc_widths)
                beam.addControlPoint(IMRTControlPoint(beam.iso, mu * total_mu, m, ga, ca, ta, xjaws, yjaws))
                if hasattr(cp, "GantryAngle"):
                    ga = cp.GantryAngle
                if hasattr(cp, "BeamLimitingDevicePositionSequence"):
                    xjaws, yjaws, mlc = read_devices(cp)
                cumulative_mu = cp.CumulativeMetersetWeight
            self.addBeam(beam)
