"""B200-native lattice Metropolis engine: the hot path of the scamper
workspace's classical Monte Carlo crate (Ising, q-state Potts, O(3) and
64-replica multi-spin Ising on periodic square and cubic lattices, with
device-side parallel tempering), behind the C ABI in include/gpumc.h.

The CUDA library (libgpumc.so, sm_100a) is the only compute path: importing
the package fails loudly if it has not been built.
"""
from . import _lib
from . import autotune
from ._lib import GpumcError, InvalidConfig
from .measurements import Accumulator, Context, Estimate, binder_cumulant, specific_heat
from .mc import (ClassicalMC, Engine, MultiSpinIsing, Params, Server, geometric_ladder_betas,
                 plan_tiles, potts_beta_c, run_one)
from .results import Metadata, Results
from .snapshot import CheckpointCorrupted

_lib.load()

__all__ = [
    "Accumulator", "CheckpointCorrupted", "ClassicalMC", "Context", "Engine", "Estimate", "GpumcError", "InvalidConfig",
    "Metadata", "MultiSpinIsing", "Params", "Results", "Server", "binder_cumulant", "geometric_ladder_betas",
    "plan_tiles", "potts_beta_c",
    "run_one", "specific_heat",
]
