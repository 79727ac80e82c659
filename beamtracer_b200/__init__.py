"""beamtracer-b200: the Vlasov iteration of beamtracer, native to the NVIDIA B200.

The reference's public interface for its self-consistent steady-beam solve --
``BeamOptics(config).run()``, ``BeamOpticsConfig`` and its sections, ``beam_moments()``,
the solver-level ``vlasov_iterate``, ``BeamTracer``, ``IonOpticsPoisson`` and the kernel
catalogue ``KERNELS`` -- over hand-written sm_100a CUDA kernels (``libbt200.so``) called
through a C ABI (``include/bt200.h``) with ctypes.  There is no CPU fallback.
"""

from beamtracer_b200.config import (
    BeamOpticsConfig,
    BeamSpecies,
    ExtractionPlasma,
    FieldBCs,
    FieldBoundaryCondition,
    GridParams,
    NegativeExtractionPlasma,
    ObjectParams,
    ParticleBeam,
    RefinementParams,
    Solenoid,
    SpaceChargeCompensation,
)
from beamtracer_b200.diagnostics import BeamMoments, mismatch, plane_moments
from beamtracer_b200.mesh import Electrode, FaceCondition, IonOpticsMesh
from beamtracer_b200.model import BeamOptics

__version__ = "0.1.0"

__all__ = [
    "BeamMoments",
    "BeamOptics",
    "BeamOpticsConfig",
    "BeamSpecies",
    "Electrode",
    "ExtractionPlasma",
    "FaceCondition",
    "FieldBCs",
    "FieldBoundaryCondition",
    "GridParams",
    "IonOpticsMesh",
    "NegativeExtractionPlasma",
    "ObjectParams",
    "ParticleBeam",
    "RefinementParams",
    "Solenoid",
    "SpaceChargeCompensation",
    "mismatch",
    "plane_moments",
]
