"""wdsgpu_b200: B200-native batched GGA (EPANET hydraulics) and implicit
adjoint, a drop-in for the batched route of the `dgga` package.

    from wdsgpu_b200 import GGASolver, implicit_solve, Net, synth
"""
from .net import Net
from . import synth

__all__ = ["Net", "synth", "GGASolver", "implicit_solve"]


def __getattr__(name):
    # the solver pulls in torch and the CUDA library lazily
    if name == "GGASolver":
        from .solver import GGASolver
        return GGASolver
    if name == "implicit_solve":
        from .autodiff import implicit_solve
        return implicit_solve
    raise AttributeError(name)
