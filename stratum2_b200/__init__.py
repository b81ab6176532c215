"""B200-native path-tracing hot path of Stratum2: wavefront path tracing with NEE and ReSTIR DI
behind a C ABI (include/stratum2.h), with sm_100a CUDA kernels in csrc/."""
from ._abi import S2Error
from .api import Device, rays_array
from .scene import Material, Scene, make_view

__all__ = ["Device", "Scene", "Material", "S2Error", "make_view", "rays_array"]
