"""attract_b200: the ATTRACT grid/neighbour-grid scoring and rigid-body ADAM
minimisation path of sjdv1982/attract-jax, as hand-written sm_100a CUDA
kernels behind a C ABI (include/attract_b200.h), driven from PyTorch.

Public API
----------
ForceField, GridGeom, Grid, LigandSet       -- inputs resident on the GPU
Workload, Segment                           -- what one launch serves
energrad, minimise, energrad_backward       -- the scoring kernels' entry points
minimise_schema                             -- the reference's quaternion/adabelief protocol, fused
MinimisePlan                                -- a graph-capturable batched minimisation
EvalOptions, AdamOptions, LaunchShape       -- options
"""
from ._lib import AttractError, load as load_library
from .engine import (AdamOptions, EvalOptions, LaunchShape, MinimisePlan, MinimiseScratch, Segment, Workload,
                     energrad, energrad_backward, minimise, minimise_schema)
from .forcefield import ForceField
from .grid import Grid, GridGeom
from .ligand import LigandSet

__all__ = ["AttractError", "load_library", "AdamOptions", "EvalOptions", "LaunchShape", "MinimisePlan",
           "MinimiseScratch", "Segment", "Workload", "energrad", "energrad_backward", "minimise", "minimise_schema",
           "ForceField",
           "Grid", "GridGeom", "LigandSet"]
