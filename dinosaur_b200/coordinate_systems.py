"""Horizontal + vertical coordinates (shape contract of
dinosaur/coordinate_systems.py:84-199; the sharding parts are not part of this
single-GPU build)."""

from __future__ import annotations

import dataclasses
from typing import Any

from dinosaur_b200 import spherical_harmonic
from dinosaur_b200 import sigma_coordinates


@dataclasses.dataclass(frozen=True)
class CoordinateSystem:
  horizontal: spherical_harmonic.Grid
  vertical: sigma_coordinates.SigmaCoordinates
  spmd_mesh: Any = None

  def __post_init__(self):
    if self.spmd_mesh is not None:
      raise NotImplementedError('spmd_mesh is not supported by this build')

  @property
  def nodal_shape(self):
    return (self.vertical.layers,) + self.horizontal.nodal_shape

  @property
  def modal_shape(self):
    return (self.vertical.layers,) + self.horizontal.modal_shape

  @property
  def surface_nodal_shape(self):
    return (1,) + self.horizontal.nodal_shape

  @property
  def surface_modal_shape(self):
    return (1,) + self.horizontal.modal_shape

  @property
  def dycore_sharding(self):
    return None
