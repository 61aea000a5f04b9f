"""B200-native evolver for GFTEvolver's real-time SU(2) x U(1) + Higgs lattice dynamics.

The hot path is the leapfrog time step of ``Lattice::evolve``
(GFTEvolver ``Core/Source/Lattice.cpp:755-876``), implemented as hand-written
sm_100a CUDA kernels behind the C ABI of ``include/gft.h``
(``libgft_b200.so``, built in-tree by ``gftevolver_b200/build.py``).
"""
from ._lib import (GFT_FORM_FP64, GFT_FORM_MIXED, GFT_FORM_REF, GFT_MODEL_2HDM, GFT_MODEL_SM, GftError,  # noqa: F401
                   load)
from .ensemble import Ensemble, ShardedEnsemble, member_shard  # noqa: F401
from .evolver import FORMS, Evolver, InitialData, LatticeParams  # noqa: F401

__all__ = ["Evolver", "Ensemble", "ShardedEnsemble", "member_shard", "LatticeParams", "InitialData", "FORMS", "GftError", "load",
           "GFT_MODEL_SM", "GFT_MODEL_2HDM", "GFT_FORM_REF", "GFT_FORM_FP64", "GFT_FORM_MIXED"]
