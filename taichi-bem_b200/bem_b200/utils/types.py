"""Enumerations with the reference's names and values
(src/BEM_functions/utils/types.py:4-57)."""
from enum import IntEnum


class CellFluxType(IntEnum):
    NEUMANN_TOBESOLVED = 0
    DIRICHLET_TOBESOLVED = 1
    MIX_NONRESOLVED = 2
    BOTH_TOBESOLVED = 3


class ScopeType(IntEnum):
    NOT_DEFINED = 0
    INTERIOR = 1
    EXTERIOR = 2


class VertAttachType(IntEnum):
    NEUMANN_TOBESOLVED = 0
    DIRICHLET_TOBESOLVED = 1
    BOTH_TOBESOLVED = 2


class KernelType(IntEnum):
    LAPLACE = 0
    HELMHOLTZ = 1
    HELMHOLTZ_TRANSMISSION = 2


class PanelsRelation(IntEnum):
    SEPARATE = 0
    COINCIDE = 1
    COMMON_VERTEX = 2
    COMMON_EDGE = 3


class AssembleType(IntEnum):
    NOTHING = 0
    ADD_HALF_IDENTITY = 1
    ADD_M = 2
    ADD_P_PLUS = 3
    ADD_P_MINUS = 4
