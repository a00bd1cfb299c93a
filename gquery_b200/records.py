"""Result records with the field names of gQuery's dataclasses
(gquery/shapes/primitive.py:10-84).

Fields are torch tensors on the scene's device, structure-of-arrays like DrJit's
Array2f/Array3f: vectors are ``[D, n]``, scalars ``[n]``, booleans ``torch.bool``,
indices ``torch.int32``.  A miss is an all-zero record (``valid`` False), as
produced by ``dr.zeros`` in the reference.
"""
from __future__ import annotations

from dataclasses import dataclass

import torch


@dataclass
class Intersection:  # primitive.py:10-17
    valid: torch.Tensor
    p: torch.Tensor
    n: torch.Tensor
    t: torch.Tensor
    d: torch.Tensor
    prim_id: torch.Tensor
    on_boundary: torch.Tensor


@dataclass
class Intersection3D:  # primitive.py:21-28
    valid: torch.Tensor
    p: torch.Tensor
    n: torch.Tensor
    uv: torch.Tensor
    d: torch.Tensor
    prim_id: torch.Tensor
    on_boundary: torch.Tensor


@dataclass
class ClosestPointRecord:  # primitive.py:32-38
    valid: torch.Tensor
    p: torch.Tensor
    n: torch.Tensor
    t: torch.Tensor
    d: torch.Tensor
    prim_id: torch.Tensor


@dataclass
class ClosestPointRecord3D:  # primitive.py:42-48
    valid: torch.Tensor
    p: torch.Tensor
    n: torch.Tensor
    uv: torch.Tensor
    d: torch.Tensor
    prim_id: torch.Tensor


@dataclass
class ClosestSilhouettePointRecord:  # primitive.py:72-76
    valid: torch.Tensor
    p: torch.Tensor
    d: torch.Tensor
    prim_id: torch.Tensor


@dataclass
class ClosestSilhouettePointRecord3D:  # primitive.py:80-84
    valid: torch.Tensor
    p: torch.Tensor
    d: torch.Tensor
    prim_id: torch.Tensor
