"""Determinant batches for the neural models.

Mirrors detnqs/utils/det_utils.py (DetBatch, BatchSpec, get_batch_spec,
prepare_batch) over ``core.prepare_det_batch``, which computes the features
on the GPU.  Host bitstrings give numpy arrays; CUDA-tensor bitstrings give
CUDA tensors on the same device, so a batch that is already resident never
crosses to the host.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any

import numpy as np

from . import core


@dataclass
class DetBatch:
    """occ int32[B, n_e] and the optional fields in aux (k, phase, holes,
    parts, hp_mask, holes_pos, parts_pos)."""

    occ: Any
    aux: dict[str, Any] = field(default_factory=dict)

    def __len__(self) -> int:
        return int(self.occ.shape[0])

    def __getitem__(self, idx) -> "DetBatch":
        return DetBatch(occ=self.occ[idx], aux={k: v[idx] for k, v in self.aux.items()})


@dataclass(frozen=True)
class BatchSpec:
    """What a model needs (det_utils.py:47-63): need_k, hp_kmax (0 = no
    hole/particle lists), need_phase, need_hp_pos."""

    need_k: bool = False
    hp_kmax: int = 0
    need_phase: bool = False
    need_hp_pos: bool = False


def get_batch_spec(model: Any) -> BatchSpec:
    """model.batch_spec, or the default spec when the model has none."""
    spec = getattr(model, "batch_spec", None)
    if spec is None:
        return BatchSpec()
    if not isinstance(spec, BatchSpec):
        raise TypeError(f"model.batch_spec must be BatchSpec, got {type(spec)}")
    return spec


def prepare_batch(bitstrings, *, n_orb: int, n_alpha: int, n_beta: int, ref,
                  spec: BatchSpec, device: int = 0) -> DetBatch:
    """DetBatch of (B, 2) alpha/beta bitstrings (det_utils.py:77-150)."""
    on_dev = hasattr(bitstrings, "is_cuda") and bitstrings.is_cuda
    dets = bitstrings if on_dev else np.asarray(bitstrings, dtype=np.uint64)
    if dets.ndim != 2 or dets.shape[1] != 2:
        raise ValueError(f"bitstrings must be (B, 2), got {tuple(dets.shape)}")
    ref = np.asarray(ref, dtype=np.uint64).reshape(-1)
    if ref.shape != (2,):
        raise ValueError(f"ref must be (2,), got {ref.shape}")
    if spec.need_hp_pos and spec.hp_kmax <= 0:
        raise ValueError("need_hp_pos requires hp_kmax > 0")
    need_hp = spec.hp_kmax > 0
    need_k = spec.need_k or need_hp
    out = core.prepare_det_batch(dets, ref, int(n_orb), int(n_alpha), int(n_beta),
                                 int(spec.hp_kmax), bool(need_k), bool(spec.need_phase),
                                 bool(need_hp), bool(spec.need_hp_pos), device=device)
    aux = {k: out[k] for k in ("k", "phase", "holes", "parts", "hp_mask", "holes_pos",
                               "parts_pos") if k in out}
    return DetBatch(occ=out["occ"], aux=aux)


__all__ = ["DetBatch", "BatchSpec", "get_batch_spec", "prepare_batch"]
