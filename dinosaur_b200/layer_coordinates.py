"""Vertical coordinate of the multi-layer shallow-water equations
(dinosaur/layer_coordinates.py:23-44)."""

from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass(frozen=True)
class LayerCoordinates:
  """Discrete constant-density layers, indexed from the top."""

  layers: int

  @property
  def centers(self) -> np.ndarray:
    return np.arange(self.layers)

  def asdict(self):
    return dataclasses.asdict(self)
