"""Base plan / dose-grid API (mirror of DoseCUDA/plan.py).

Same classes, attributes and method names as the reference.  The CT/dose
file readers and writers (NRRD, NIfTI, DICOM) need SimpleITK / pydicom; they
are imported only inside those methods, so the dose path runs without them.
"""
from __future__ import annotations

import numpy as np


def _sitk():
    try:
        import SimpleITK as sitk  # noqa: N813
    except ImportError as e:  # pragma: no cover - depends on the environment
        raise ImportError("this method reads/writes image files and needs SimpleITK") from e
    return sitk


def _pydicom():
    try:
        import pydicom
    except ImportError as e:  # pragma: no cover - depends on the environment
        raise ImportError("this method reads/writes DICOM and needs pydicom") from e
    return pydicom


class VolumeObject:
    """Attribute bag handed to the dose kernels (reference plan.py:6-11)."""

    def __init__(self):
        self.origin = np.array([0.0, 0.0, 0.0], dtype=np.single)
        self.spacing = np.array([0.0, 0.0, 0.0], dtype=np.single)
        self.voxel_data = []


class DoseGrid:
    """CT grid plus the computed dose (reference plan.py:14-224).

    ``HU`` and ``dose`` are numpy arrays of shape (nz, ny, nx); ``origin`` and
    ``spacing`` are in (x, y, z) order, mm."""

    def __init__(self):
        self.origin = np.array([0.0, 0.0, 0.0], dtype=np.single)
        self.spacing = np.array([0.0, 0.0, 0.0], dtype=np.single)
        self.size = np.array([0, 0, 0])
        self.HU = []
        self.dose = []
        self.beam_doses = []
        self.FrameOfReferenceUID = ""

    # -- synthetic phantoms -------------------------------------------------
    def createCubePhantom(self, size=[138, 138, 138], spacing=3.0):  # noqa: B006 (reference signature)
        """Water cube in air with a 10 mm air margin (reference plan.py:218-224)."""
        self.origin = np.array([-size[0] * spacing / 2.0, -size[1] * spacing / 2.0, -size[2] * spacing / 2.0])
        self.spacing = np.array([spacing, spacing, spacing])
        self.size = np.array(size)
        edge = round(10.0 / spacing)
        self.HU = np.ones(size, dtype=np.single) * -1000.0
        self.HU[edge:-edge, edge:-edge, edge:-edge] = 0.0

    def applyCouchModel(self, couch_wet=8.0):
        """Override the posterior 50 mm with a uniform couch of the given WET
        (reference plan.py:118-123)."""
        spacing = self.spacing[0]
        n_voxels = int(50.0 / spacing)
        hu_override_value = ((couch_wet / (n_voxels * spacing)) - 1.0) * 1000.0
        self.HU[:, -n_voxels:, :] = hu_override_value

    # -- file I/O (needs SimpleITK / pydicom) -------------------------------
    def loadCTNRRD(self, ct_path):
        sitk = _sitk()
        fr = sitk.ImageFileReader()
        fr.SetFileName(ct_path)
        img = fr.Execute()
        self.origin = np.array(img.GetOrigin())
        self.spacing = np.array(img.GetSpacing())
        self.HU = np.array(sitk.GetArrayFromImage(img), dtype=np.single)
        self.size = np.array(self.HU.shape)

    def loadCTDCM(self, ct_path):
        sitk = _sitk()
        pyd = _pydicom()
        reader = sitk.ImageSeriesReader()
        names = list(reader.GetGDCMSeriesFileNames(ct_path))
        names.sort(key=lambda x: pyd.dcmread(x, force=True).ImagePositionPatient[2])
        reader.SetFileNames(names)
        img = reader.Execute()
        self.origin = np.array(img.GetOrigin())
        self.spacing = np.array(img.GetSpacing())
        self.HU = np.clip(np.array(sitk.GetArrayFromImage(img), dtype=np.single), -1000.0, None)
        self.size = np.array(self.HU.shape)

    def _resample(self, rf):
        sitk = _sitk()
        img = sitk.GetImageFromArray(self.HU)
        img.SetOrigin(self.origin)
        img.SetSpacing(self.spacing)
        rf.SetDefaultPixelValue(-1000)
        return np.array(sitk.GetArrayFromImage(rf.Execute(img)), dtype=np.single)

    def resampleCT(self, new_spacing, new_size, new_origin):
        sitk = _sitk()
        rf = sitk.ResampleImageFilter()
        rf.SetOutputOrigin(new_origin)
        rf.SetOutputSpacing(new_spacing)
        rf.SetSize(new_size)
        self.HU = self._resample(rf)
        self.origin = new_origin
        self.spacing = new_spacing
        self.size = np.array(self.HU.shape)

    def resampleCTfromSpacing(self, spacing):
        sitk = _sitk()
        rf = sitk.ResampleImageFilter()
        rf.SetOutputOrigin(self.origin)
        sp_new = (spacing, spacing, spacing)
        sz_new = (int(self.size[2] * self.spacing[0] / sp_new[0]),
                  int(self.size[1] * self.spacing[1] / sp_new[1]),
                  int(self.size[0] * self.spacing[2] / sp_new[2]))
        rf.SetOutputSpacing(sp_new)
        rf.SetSize(sz_new)
        self.HU = self._resample(rf)
        self.spacing = sp_new
        self.size = np.array(self.HU.shape)

    def resampleCTfromReferenceDose(self, ref_dose_path):
        sitk = _sitk()
        pyd = _pydicom()
        ref = pyd.dcmread(ref_dose_path, force=True)
        dz = float(ref.GridFrameOffsetVector[1]) - float(ref.GridFrameOffsetVector[0])
        ref_spacing = np.array([float(ref.PixelSpacing[0]), float(ref.PixelSpacing[1]), dz])
        ref_origin = np.array(ref.ImagePositionPatient)
        ref_img = sitk.GetImageFromArray(ref.pixel_array)
        ref_img.SetOrigin(ref_origin)
        ref_img.SetSpacing(ref_spacing)
        rf = sitk.ResampleImageFilter()
        rf.SetReferenceImage(ref_img)
        self.HU = self._resample(rf)
        self.size = np.array(self.HU.shape)
        self.origin = ref_origin
        self.spacing = ref_spacing

    @staticmethod
    def _rbe(dose_type):
        if dose_type == "EFFECTIVE":
            return 1.1
        if dose_type == "PHYSICAL":
            return 1.0
        raise Exception("Unknown dose type: %s" % dose_type)

    def writeDoseDCM(self, dose_path, ref_dose_path, dose_type="EFFECTIVE", individual_beams=False):
        if not dose_path.endswith(".dcm"):
            raise Exception("Dose path must have .dcm extension")
        pyd = _pydicom()
        rbe = self._rbe(dose_type)

        def write(dose, path, summation):
            ref = pyd.dcmread(ref_dose_path)
            ref.SeriesDescription = ref.SeriesDescription + "_DoseCUDA"
            ref.DoseSummationType = summation
            ref.DoseType = dose_type
            ref.ReferencedRTPlanSequence[0].ReferencedSOPInstanceUID = pyd.uid.generate_uid()
            ref.PixelData = np.array(dose * 500.0 * rbe, dtype=np.uint16)
            ref.DoseGridScaling = 0.002
            ref.save_as(path)

        if individual_beams:
            for i, bd in enumerate(self.beam_doses):
                write(bd, dose_path.replace(".dcm", "_beam%02i.dcm" % (i + 1)), "BEAM")
        else:
            write(self.dose, dose_path, "PLAN")

    def writeDoseNRRD(self, dose_path, individual_beams=False, dose_type="EFFECTIVE"):
        if not dose_path.endswith(".nrrd"):
            raise Exception("Dose path must have .nrrd extension")
        rbe = self._rbe(dose_type)
        sitk = _sitk()
        fw = sitk.ImageFileWriter()

        def image(d):
            img = sitk.GetImageFromArray(np.array(d * rbe, dtype=np.single))
            img.SetOrigin(self.origin)
            img.SetSpacing(self.spacing)
            return img

        if individual_beams:
            for i, bd in enumerate(self.beam_doses):
                fw.SetFileName(dose_path.replace(".nrrd", "_beam%02i.nrrd" % (i + 1)))
                fw.Execute(image(bd))
        else:
            fw.SetFileName(dose_path)
            fw.Execute(image(self.dose))

    def _write_ct(self, path):
        sitk = _sitk()
        img = sitk.GetImageFromArray(self.HU)
        img.SetOrigin(self.origin)
        img.SetSpacing(self.spacing)
        fw = sitk.ImageFileWriter()
        fw.SetFileName(path)
        fw.Execute(img)

    def writeCTNRRD(self, ct_path):
        if not ct_path.endswith(".nrrd"):
            raise Exception("CT path must have .nrrd extension")
        self._write_ct(ct_path)

    def writeCTNIFTI(self, ct_path):
        if not ct_path.endswith(".nii.gz"):
            raise Exception("CT path must have .nii.gz extension")
        self._write_ct(ct_path)


class Beam:
    def __init__(self):
        self.iso = np.array([0.0, 0.0, 0.0], dtype=np.single)
        self.gantry_angle = 0.0
        self.collimator_angle = 0.0
        self.couch_angle = 0.0


class Plan:
    def __init__(self):
        self.n_beams = 0
        self.n_fractions = 1
        self.beam_list = []

    def addBeam(self, beam):
        self.beam_list.append(beam)
        self.n_beams += 1
