"""Model plugin interface mirroring torch_sim/models/interface.py:71-201.

A model is a ``torch.nn.Module`` whose ``forward(state) -> dict`` returns
``energy [S]``, ``forces [N,3]`` and ``stress [S,3,3]`` (when enabled), with
``device``, ``dtype``, ``compute_forces``, ``compute_stress`` and
``memory_scales_with`` properties.  Outputs are detached and the input state is
never mutated (interface.py:354-384, 475-483).
"""

from __future__ import annotations

import torch


class ModelInterface(torch.nn.Module):
    _device: torch.device
    _dtype: torch.dtype
    _compute_stress: bool = False
    _compute_forces: bool = True
    _memory_scales_with: str = "n_atoms_x_density"

    @property
    def device(self) -> torch.device:
        return self._device

    @property
    def dtype(self) -> torch.dtype:
        return self._dtype

    @property
    def compute_stress(self) -> bool:
        return self._compute_stress

    @compute_stress.setter
    def compute_stress(self, v: bool) -> None:
        self._compute_stress = bool(v)

    @property
    def compute_forces(self) -> bool:
        return self._compute_forces

    @compute_forces.setter
    def compute_forces(self, v: bool) -> None:
        self._compute_forces = bool(v)

    @property
    def memory_scales_with(self) -> str:
        return self._memory_scales_with

    def forward(self, state, **kwargs) -> dict[str, torch.Tensor]:  # pragma: no cover
        raise NotImplementedError
