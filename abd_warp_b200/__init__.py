"""B200-native affine body dynamics (ABD) implicit contact step.

A drop-in for the time step of Luke-Skycrawler/abd-warp (``AffineBodySimulator.step``,
abd/abd.py:212-276).  The Python layer mirrors the reference's API; the work runs in
``libabd_b200.so`` (hand-written sm_100a CUDA behind a C ABI, include/abd_b200.h).
"""
from .params import SimParams
from .affine_body import AffineMesh, AffineBodyStates, WarpMesh, Scene, affine_body_states_empty
from . import scenes, meshes

__all__ = ["SimParams", "AffineMesh", "AffineBodyStates", "WarpMesh", "Scene",
           "affine_body_states_empty", "scenes", "meshes"]
