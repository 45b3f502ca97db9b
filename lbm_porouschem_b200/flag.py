"""Model switches with the reference's names and values (src/LBM/util/flag.py:10-110),
so that code written against the reference's solver keeps working."""
from enum import Enum


class VISCOSITY_MODEL(Enum):
    NONE = 0
    CONSTANT = 1
    SUTHERLAND = 2
    MIXTURE = 3


class PORO_MODEL(Enum):
    SPHERICAL = 0
    DARCY = 1
    DARCYFORCHHEIMER = 2
    DARCY_HIGH = 3
    ERGUN = 4


class CONDUCTIVITY_MODEL(Enum):
    NONE = 0
    CONSTANT = 1
    POLYNOMIAL = 2
    MIXTURE = 3


class THERMO_MODEL(Enum):
    NONE = 0
    CONSTANT = 1
    POLYNOMIAL = 2
    NASA7 = 3
    MIXTURE = 4


class THERMAL_DIFF_MODEL(Enum):
    NONE = 0
    CONSTANT = 1
    DERIVED = 2
    PRANDTL = 3


class FLUID_STATE_EQUATION(Enum):
    IDEAL_GAS = 0
    INCOMPRESSIBLE = 1


class RADIATION_MODEL(Enum):
    NONE = 0
    SURFACE_UNIFORM = 1
    REAL_RADIATION = 2
    P1_APPROACH = 3


class SOURCE_TERM(Enum):
    NONE = 0
    MICRO = 1
    MACRO = 2


class FORCE_TERM(Enum):
    NONE = 0
    GUO = 1
    SHAN = 2
    MACRO = 3


class BC(Enum):
    periodic = 0
    zeroGradient = 1
    fixedValue = 2


class BC_FLOW(Enum):
    periodic = 0
    inlet = 1
    outlet = 2
    wall = 3
    symmetric = 4
    inlet_flow = 5


class BC_MODEL(Enum):
    NONE = 0
    NEE = 1
    NEBB = 2
    ES = 3
