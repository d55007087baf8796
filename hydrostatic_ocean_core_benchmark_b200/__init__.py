"""B200 (sm_100a) implementation of the hydrostatic Boussinesq ocean-core time step.

Drop-in for the reference's v0.5/v0.6 step (``Stepper3DV05``) and its backend
protocol (``<binary> <prefix>.nml``), computing bit-for-bit the reference's fp64
results. The compute path is the CUDA library ``lib/libocean_b200.so``;
importing this package never falls back to a CPU implementation.
"""

from .params import OceanParams, params_from_reference, read_namelist, write_namelist  # noqa: F401

__all__ = ["OceanParams", "params_from_reference", "read_namelist", "write_namelist",
           "OceanStepper", "Stepper3DV05", "State3D", "thomas"]


def __getattr__(name):
    if name in ("OceanStepper", "Stepper3DV05", "State3D", "thomas"):
        from . import stepper
        return getattr(stepper, name)
    raise AttributeError(name)
