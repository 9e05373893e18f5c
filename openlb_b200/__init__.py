"""openlb_b200 — a B200-native fused collide-and-stream behind OpenLB's API.

The compute path is the in-tree sm_100a library ``libolb_b200.so`` (C ABI in
``include/olb_b200.h``); this package binds it and mirrors the reference's
host-side lattice API.  There is no CPU fallback.
"""
from . import _abi, boundary
from .descriptors import D3Q19, D3Q27, Descriptor, descriptor
from .lattice import (BGKdynamics, BounceBack, BounceBackVelocity, Dynamics, ForcedBGKdynamics,
                      ForcedTRTdynamics, InterpolatedPressureBoundary, InterpolatedVelocityBoundary, Lattice,
                      LocalPressureBoundary, LocalVelocityBoundary, NoDynamics, SmagorinskyBGKdynamics, SuperGeometry, SuperLattice,
                      TRTdynamics, VelocityCornerBoundary, VelocityEdgeBoundary, VelocityInnerCornerBoundary,
                      VelocityInnerEdgeBoundary)

OlbError = _abi.OlbError
Diverged = _abi.Diverged
LibraryNotBuilt = _abi.LibraryNotBuilt


def library_path(variant: str = "fast"):
    return _abi.library_path(variant)


def build_info() -> str:
    return _abi.load().olb_b200_build_info().decode()


__all__ = [
    "D3Q19", "D3Q27", "Descriptor", "descriptor", "Dynamics", "NoDynamics", "BGKdynamics",
    "TRTdynamics", "ForcedTRTdynamics", "ForcedBGKdynamics", "SmagorinskyBGKdynamics", "BounceBack",
    "BounceBackVelocity", "InterpolatedVelocityBoundary", "InterpolatedPressureBoundary",
    "LocalVelocityBoundary", "LocalPressureBoundary", "VelocityEdgeBoundary", "VelocityCornerBoundary", "VelocityInnerEdgeBoundary",
    "VelocityInnerCornerBoundary", "boundary",
    "Lattice", "SuperGeometry", "SuperLattice", "OlbError", "Diverged",
    "LibraryNotBuilt", "library_path", "build_info",
]
