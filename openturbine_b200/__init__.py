"""B200-native per-step beam path of Kynema (formerly Exawind/openturbine).

The compute path is the CUDA library ``libkynema_b200.so`` (sm_100a) behind the
C ABI declared in ``include/kynema_b200.h``; ``openturbine_b200.runtime`` loads
it and raises if it is missing.  ``openturbine_b200.model`` mirrors the
reference's host-side Model builder.
"""
from .model import (  # noqa: F401
    BeamSection,
    CreateTrapezoidalQuadrature,
    GaussLegendreQuadrature,
    GenerateGLLPoints,
    Model,
    QuaternionCompose,
    RotateVectorByQuaternion,
    RotationVectorToQuaternion,
    StepParameters,
)
