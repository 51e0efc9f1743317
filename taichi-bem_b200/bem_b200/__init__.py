"""bem_b200: Galerkin BEM on one NVIDIA B200 (sm_100a), a drop-in for the
operator and driver surface of GeCao/taichi-BEM (``src/managers``,
``src/BEM_functions``).  Hot paths run in libbem_b200.so (hand-written CUDA)
behind the C ABI in include/bem_b200.h."""
from . import _lib
from .meshes import analytical_disk, analytical_sphere, icosphere, load_obj, perturbed_sphere

__all__ = ["_lib", "analytical_disk", "analytical_sphere", "icosphere", "load_obj", "perturbed_sphere"]
