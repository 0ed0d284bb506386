"""inti_b200 — B200 (sm_100a) Nyström operator application for Inti.jl's
integral operators, behind a host mirror of Inti's operator API.

The compute path is libinti_b200.so (CUDA, built by inti.jl_b200/build.py);
this package is the host side: geometry/quadrature setup and ctypes calls
into the C ABI declared in include/inti_b200.h.
"""
from . import _lib
from ._lib import (
    ArgumentError,
    DeviceError,
    DimensionMismatch,
    InticError,
    NonFiniteError,
    UnsupportedError,
)
from .core import *  # noqa: F401,F403
from .core import __all__ as _core_all
from .vdim import polynomial_solutions_vdim, vdim_correction
from .autodiff import TorchPotential, rrule
from .geometry import (
    Quadrature,
    circle_quadrature,
    curve_quadrature,
    ball_hex_quadrature,
    disk_triangle_quadrature,
    ellipsoid_quadrature,
    gauss_legendre,
    kite_quadrature,
    p2_sphere_quadrature,
    points,
    star_coefficients,
    star_quadrature,
)

__all__ = list(_core_all) + [
    "Quadrature",
    "points",
    "kite_quadrature",
    "circle_quadrature",
    "curve_quadrature",
    "ball_hex_quadrature",
    "disk_triangle_quadrature",
    "ellipsoid_quadrature",
    "p2_sphere_quadrature",
    "star_quadrature",
    "star_coefficients",
    "gauss_legendre",
    "polynomial_solutions_vdim",
    "vdim_correction",
    "rrule",
    "TorchPotential",
    "ArgumentError",
    "DimensionMismatch",
    "NonFiniteError",
    "UnsupportedError",
    "DeviceError",
    "InticError",
]
