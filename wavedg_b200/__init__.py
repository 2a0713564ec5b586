"""wavedg_b200: the 2D wave DG hot path of waveDG on B200 (sm_100a).

The product is the C-ABI library ``libwdg_b200.so`` (include/wdg_b200.h);
this package is its Python mirror of the reference's ``dg::`` classes.
"""
from ._lib import WDG_FP32, WDG_FP64, WdgError, lib  # noqa: F401
from .dg import (  # noqa: F401
    Advection,
    AdvectionHomogeneousBC,
    AdvectionSystem,
    Discretisation,
    Div,
    ExactDiscretisation,
    EdgeFlux,
    EulerSystem,
    VariableAdvectionSystem,
    BasisMassMatrix,
    FaceProlongator,
    FaceType,
    LinearFunctional2D,
    MassMatrix,
    Mesh2D,
    Operator,
    QuadratureRule,
    RungeKutta4,
    WaveBC,
    WaveEquation,
    WaveHoltz,
    WaveHoltzBatch,
    WaveSystem,
    error,
    make_face_prolongator,
    norm,
    read_file,
    to_file,
)

__all__ = [
    "Advection", "AdvectionHomogeneousBC", "AdvectionSystem", "read_file", "to_file", "Discretisation", "Div", "ExactDiscretisation", "EdgeFlux", "EulerSystem", "VariableAdvectionSystem", "BasisMassMatrix",
    "FaceProlongator", "FaceType", "LinearFunctional2D", "MassMatrix",
    "Mesh2D", "Operator", "QuadratureRule", "RungeKutta4", "WaveBC", "WaveEquation", "WaveHoltz", "WaveHoltzBatch", "WaveSystem",
    "WdgError", "WDG_FP32", "WDG_FP64", "error", "lib", "make_face_prolongator", "norm",
]
