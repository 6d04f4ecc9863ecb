"""DoseCUDA on B200: proton pencil-beam and photon collapsed-cone dose engines
written as hand-tuned sm_100a CUDA kernels behind the reference DoseCUDA
Python API.

    from dosecuda_b200 import IMPTDoseGrid, IMPTPlan, IMPTBeam
    from dosecuda_b200 import IMRTDoseGrid, IMRTPlan, IMRTBeam, IMRTControlPoint, IMRTPhotonEnergy

``dosecuda_b200.dose_kernels`` is the drop-in for the reference's compiled
``dose_kernels`` module; ``dosecuda_b200.engine`` is the device-resident
interface (torch CUDA tensors, explicit streams).
"""
from .plan_impt import IMPTBeam, IMPTBeamModel, IMPTDoseGrid, IMPTPlan
from .plan_imrt import IMRTBeam, IMRTControlPoint, IMRTDoseGrid, IMRTPhotonEnergy, IMRTPlan

__all__ = ["IMPTDoseGrid", "IMPTPlan", "IMPTBeam", "IMPTBeamModel", "IMRTDoseGrid", "IMRTPlan", "IMRTBeam",
           "IMRTControlPoint", "IMRTPhotonEnergy"]
