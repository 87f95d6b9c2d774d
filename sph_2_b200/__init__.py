"""sph_2_b200 -- B200-native (sm_100a) per-step hot path of a self-gravitating
SPH code: Morton sort + radix tree, exact neighbour lists, Newton smoothing
lengths, density / div-curl / force / du/dt passes with Monaghan viscosity,
a quadrupole Barnes-Hut walk, implicit cooling with an MLP surrogate, and the
leapfrog step, all as CUDA kernels behind the C ABI in include/sph_b200.h.
"""
from .core import Config, Context  # noqa: F401
from . import ic  # noqa: F401

__all__ = ["Config", "Context", "ic"]
