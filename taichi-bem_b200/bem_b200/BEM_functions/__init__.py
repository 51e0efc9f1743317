from .layers import (SingleLayer3d, DoubleLayer3d, AdjDoubleLayer3d, HypersingularLayer3d, IdentityLayer3d,
                     RHSConstructor3d)

__all__ = ["SingleLayer3d", "DoubleLayer3d", "AdjDoubleLayer3d", "HypersingularLayer3d", "IdentityLayer3d",
           "RHSConstructor3d"]
