"""diffractom_b200: diffractom's reconstruction hot path (the single-phase forward operator, its adjoint and the
SPDHG / FISTA Poisson, FISTA least-squares / Huber solvers) as hand-written sm_100a CUDA kernels behind a C ABI, with diffractom's Python API.

    from diffractom_b200 import Material, Grid, SinglePhaseForwardOperator, SPDHGPoisson

Device arrays are CUDA torch tensors (float32, contiguous) in place of pyopencl arrays; NumPy arrays are accepted
where diffractom accepts them. The CUDA library is built in-tree by `python -m diffractom_b200.build`.
"""
from .grid import Grid, MatrixGrid
from .orientation_tree import OrientationTree
from .material import Material, group_reflections_into_rings
from .quadrature import QuadratureRule

__all__ = ["Grid", "MatrixGrid", "Material", "QuadratureRule", "group_reflections_into_rings", "OrientationTree",
           "SinglePhaseForwardOperator", "SPDHGPoisson", "FISTAPoisson", "FISTAHuber", "FISTAL2", "OSEMPoisson",
           "PDHGPoisson", "estimate_L_power", "estimate_L_power_streamed",
           "forward_operator"]


def __getattr__(name):
    # the device classes import torch and the CUDA library only when used
    if name in ("SinglePhaseForwardOperator", "estimate_L_power", "estimate_L_power_streamed"):
        from . import operator
        return getattr(operator, name)
    if name == "SPDHGPoisson":
        from .spdhg import SPDHGPoisson
        return SPDHGPoisson
    if name == "FISTAPoisson":
        from .fista import FISTAPoisson
        return FISTAPoisson
    if name in ("OSEMPoisson", "PDHGPoisson"):
        from . import osem_pdhg
        return getattr(osem_pdhg, name)
    if name in ("FISTAHuber", "FISTAL2"):
        from . import fista_ls
        return getattr(fista_ls, name)
    if name == "forward_operator":
        from .autograd import forward_operator
        return forward_operator
    raise AttributeError(name)
