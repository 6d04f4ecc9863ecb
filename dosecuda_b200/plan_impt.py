"""IMPT plan API (mirror of DoseCUDA/plan_impt.py).

Class and method names, attributes and array layouts are the reference's, so
existing scripts run unchanged; the dose calls go to the sm_100a engine via
``dosecuda_b200.dose_kernels``.  DICOM reading (``readPlanDicom``) imports
pydicom lazily; the RT-Ion plan writer of the reference (plan_impt.py:307-608)
is not part of this package.
"""
from __future__ import annotations

import os

import numpy as np
import pandas as pd

from . import dose_kernels
from .lookup import read_proton_energy, table_path
from .plan import Beam, DoseGrid, Plan, VolumeObject, _pydicom


class IMPTBeamModel:
    """Proton beam model of one range-shifter setting (reference plan_impt.py:17-103).

    Attributes used by the engine: ``VSADX``, ``VSADY`` (mm),
    ``divergence_params`` [nE, 5] = energy, R80, A, B, C, and
    ``lut_depths`` / ``lut_sigmas`` / ``lut_idds`` [nE, 400], float32."""

    def __init__(self, dicom_rangeshifter_label, path_to_model, folder_rangeshifter_label):
        self.dicom_rangeshifter_label = dicom_rangeshifter_label
        self.VSADX = None
        self.VSADY = None
        with open(os.path.join(path_to_model, "machine_geometry.csv"), "r") as f:
            for line in f:
                if line.startswith("VSADX"):
                    self.VSADX = float(line.split(",")[1])
                if line.startswith("VSADY"):
                    self.VSADY = float(line.split(",")[1])
        if self.VSADX is None:
            raise Exception("VSADX not found in machine_geometry.csv")
        if self.VSADY is None:
            raise Exception("VSADY not found in machine_geometry.csv")

        folder = os.path.join(path_to_model, folder_rangeshifter_label)
        self.energy_table = pd.read_csv(os.path.join(folder, "energies.csv"))
        self.energy_labels = self.energy_table["energy_label"].to_numpy()
        energy_ids = self.energy_table["index"].to_numpy()
        self.reference_sigmas = self.energy_table["sigma"].to_numpy()

        dvp, depths, sigmas, idds = [], [], [], []
        for eid in energy_ids:
            params, rows = read_proton_energy(os.path.join(folder, "energy_%03d.csv" % eid))
            dvp.append(params)
            depths.append([r[0] for r in rows])
            sigmas.append([r[1] for r in rows])
            idds.append([r[2] for r in rows])
        self.divergence_params = np.array(dvp, dtype=np.single)
        self.lut_depths = np.array(depths, dtype=np.single)
        self.lut_sigmas = np.array(sigmas, dtype=np.single)
        self.lut_idds = np.array(idds, dtype=np.single)

    def energyIDFromLabel(self, energy_label):
        row = self.energy_table[self.energy_table["energy_label"] == energy_label]
        if len(row) != 1:
            raise Exception("Energy ID not found for %.2f" % energy_label)
        return row.index[0]


class IMPTDoseGrid(DoseGrid):
    def __init__(self):
        super().__init__()
        self.RLSP = []

    def RLSPFromHU(self, machine_name):
        """Piecewise-linear HU -> relative linear stopping power (reference
        plan_impt.py:112-122)."""
        df = pd.read_csv(table_path("protons", machine_name, "HU_RLSP.csv"))
        return np.array(np.interp(self.HU, df["HU"].to_numpy(), df["RLSP"].to_numpy()), dtype=np.single)

    def _volume(self, data):
        v = VolumeObject()
        v.voxel_data = np.array(data, dtype=np.single)
        v.origin = np.array(self.origin, dtype=np.single)
        v.spacing = np.array(self.spacing, dtype=np.single)
        return v

    def _check_isotropic(self):
        if self.spacing[0] != self.spacing[1] or self.spacing[0] != self.spacing[2]:
            raise Exception("Spacing must be isotropic for IMPT dose calculation - consider resampling CT")

    @staticmethod
    def _model_for(plan, beam):
        labels = list(plan.dicom_rangeshifter_label.astype(str))
        if beam.dicom_rangeshifter_label not in labels:
            raise ValueError("Beam model not found for rangeshifter ID %s" % beam.dicom_rangeshifter_label)
        return plan.beam_models[labels.index(beam.dicom_rangeshifter_label)]

    def computeIMPTPlan(self, plan, gpu_id=0, device=False):
        """Dose of every beam: WET ray trace then pencil-beam dose, scaled by
        the number of fractions (reference plan_impt.py:124-160).

        ``device=True`` keeps the plan on the GPU: the HU volume is uploaded
        once and converted there, straight into the ray tracer's texture;
        every beam's WET and dose stay on the device and are summed there; the
        results are copied back once.  Same arithmetic as the host loop."""
        if device:
            return self._computeIMPTPlanDevice(plan, gpu_id)
        self.beam_doses = []
        self.dose = np.zeros(self.size, dtype=np.single)
        self.RLSP = self.RLSPFromHU(plan.machine_name)
        self._check_isotropic()
        rlsp = self._volume(self.RLSP)
        for beam in plan.beam_list:
            model = self._model_for(plan, beam)
            wet = self._volume(dose_kernels.proton_raytrace_cuda(model, rlsp, beam, gpu_id))
            beam_dose = dose_kernels.proton_spot_cuda(model, rlsp, wet, beam, gpu_id)
            self.beam_doses.append(beam_dose * plan.n_fractions)
            self.dose += beam_dose
        self.dose *= plan.n_fractions

    def _computeIMPTPlanDevice(self, plan, gpu_id):
        import torch

        from . import engine
        self._check_isotropic()
        dev = torch.device("cuda", gpu_id)
        df = pd.read_csv(table_path("protons", plan.machine_name, "HU_RLSP.csv"))
        table = (df["HU"].to_numpy(), df["RLSP"].to_numpy())
        hu = torch.as_tensor(np.ascontiguousarray(self.HU, dtype=np.single), device=dev)
        total = torch.zeros(hu.shape, dtype=torch.float32, device=dev)
        doses, dmodels = [], {}
        for beam in plan.beam_list:
            model = self._model_for(plan, beam)
            if id(model) not in dmodels:
                dmodels[id(model)] = engine.ProtonModelDevice(model, device=dev)
            wet = engine.proton_wet_hu(hu, self, beam, model, table)
            beam_dose = engine.proton_dose(wet, self, beam, dmodels[id(model)])
            doses.append(beam_dose * plan.n_fractions)
            total += beam_dose
        total *= plan.n_fractions
        self.RLSP = engine.hu_convert(hu, table).cpu().numpy()
        self.beam_doses = [d.cpu().numpy() for d in doses]
        self.dose = total.cpu().numpy()

    def computeIMPTWET(self, plan, gpu_id=0):
        """Per-beam smoothed WET volumes, for reuse across spot-weight changes
        (reference plan_impt.py:162-190)."""
        self.RLSP = self.RLSPFromHU(plan.machine_name)
        rlsp = self._volume(self.RLSP)
        out = []
        for beam in plan.beam_list:
            model = self._model_for(plan, beam)
            out.append(self._volume(dose_kernels.proton_raytrace_cuda(model, rlsp, beam, gpu_id)))
        return out

    def computeIMPTPlanFromWET(self, plan, wet_object, beam, gpu_id=0):
        """One beam's dose from a precomputed WET (reference plan_impt.py:192-211)."""
        self._check_isotropic()
        rlsp = self._volume(self.RLSP)
        model = self._model_for(plan, beam)
        return dose_kernels.proton_spot_cuda(model, rlsp, wet_object, beam, gpu_id)

    def writeWETNRRD(self, plan, wet_path, gpu_id=0):
        if not wet_path.endswith(".nrrd"):
            raise Exception("WET path must have .nrrd extension")
        from .plan import _sitk
        sitk = _sitk()
        self.RLSP = self.RLSPFromHU(plan.machine_name)
        rlsp = self._volume(self.RLSP)
        fw = sitk.ImageFileWriter()
        for i, beam in enumerate(plan.beam_list):
            wet = dose_kernels.proton_raytrace_cuda(self._model_for(plan, beam), rlsp, beam, gpu_id)
            img = sitk.GetImageFromArray(wet)
            img.SetOrigin(self.origin)
            img.SetSpacing(self.spacing)
            fw.SetFileName(wet_path.replace(".nrrd", "_beam%02i.nrrd" % (i + 1)))
            fw.Execute(img)


class IMPTBeam(Beam):
    """Spot-scanning beam.  ``spot_list`` is an (n, 4) float32 array of
    x (mm), y (mm), MU, energy id (reference plan_impt.py:244-281)."""

    def __init__(self, beam=None):
        super().__init__()
        self.spot_list = []
        self.n_spots = 0
        self.dicom_rangeshifter_label = None
        if beam is not None:
            self.gantry_angle = beam.gantry_angle
            self.couch_angle = beam.couch_angle
            self.iso = beam.iso
            self.spot_list = beam.spot_list
            self.n_spots = beam.n_spots
            self.dicom_rangeshifter_label = beam.dicom_rangeshifter_label

    def addSpotData(self, cp, energy_id):
        spm = np.reshape(np.array(cp.ScanSpotPositionMap), (-1, 2))
        mus = np.array(cp.ScanSpotMetersetWeights)
        spots = np.array(np.column_stack((spm, mus, np.full(mus.size, energy_id))), dtype=np.single)
        self.spot_list = np.vstack((self.spot_list, spots)) if self.n_spots > 0 else spots
        self.n_spots += mus.size

    def changeSpotEnergy(self, energy_id):
        self.spot_list[:, 3] = energy_id

    def addSingleSpot(self, x, y, mu, energy_id):
        # Kept 2-D from the first spot on (the reference stores a 1-D row for a
        # single spot, which its own dose call then rejects).
        spot = np.array([[x, y, mu, energy_id]], dtype=np.single)
        self.spot_list = np.vstack((self.spot_list, spot)) if self.n_spots > 0 else spot
        self.n_spots += 1

    def resetSpots(self):
        self.spot_list = np.empty((0, 4), dtype=np.single)
        self.n_spots = 0


class IMPTPlan(Plan):
    def __init__(self, machine_name="HitachiProbeatJHU"):
        super().__init__()
        self.machine_name = machine_name
        model_dir = table_path("protons", machine_name)
        rs = pd.read_csv(os.path.join(model_dir, "rangeshifter_labels.csv"))
        self.dicom_rangeshifter_label = rs["dicom_rangeshifter_label"]
        self.folder_rangeshifter_label = rs["folder_rangeshifter_label"]
        self.beam_models = [IMPTBeamModel(d, model_dir, f)
                            for d, f in zip(self.dicom_rangeshifter_label, self.folder_rangeshifter_label)]

    def load_ct_series(self, ct_dir):
        pyd = _pydicom()
        files = [os.path.join(ct_dir, f) for f in os.listdir(ct_dir) if f.lower().endswith(".dcm")]
        dsets = [pyd.dcmread(f) for f in files]
        dsets.sort(key=lambda ds: ds.InstanceNumber)
        return dsets

    def readPlanDicom(self, plan_path):
        """Spot lists of an RT Ion Plan (reference plan_impt.py:610-643)."""
        pyd = _pydicom()
        ds = pyd.dcmread(plan_path, force=True)
        self.n_fractions = float(ds.FractionGroupSequence[0].NumberOfFractionsPlanned)
        self.beam_list = []
        self.n_beams = 0
        for ibs in ds.IonBeamSequence:
            beam = IMPTBeam()
            if ibs.NumberOfRangeShifters and ibs.RangeShifterSequence[0].RangeShifterID is not None:
                beam.dicom_rangeshifter_label = ibs.RangeShifterSequence[0].RangeShifterID
            else:
                beam.dicom_rangeshifter_label = "0"
            cp0 = ibs.IonControlPointSequence[0]
            beam.gantry_angle = float(cp0.GantryAngle)
            beam.couch_angle = float(cp0.PatientSupportAngle)
            beam.iso = np.array(cp0.IsocenterPosition, dtype=np.single)
            for j, cp in enumerate(ibs.IonControlPointSequence):
                if j % 2 == 0:
                    beam.addSpotData(cp, self.beam_models[0].energyIDFromLabel(float(cp.NominalBeamEnergy)))
            self.addBeam(beam)
