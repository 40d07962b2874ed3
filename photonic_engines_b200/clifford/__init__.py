"""Exact Clifford & Clifford Fock sampler on B200 (arXiv:1706.01260, arXiv:2005.04214).

    fock_sample(U, in_modes, shots, generator, loss=, indist=, ...)   the reference's entry point
    emitter_sample(EmitterMPS, U, shots, generator)                    EmitterMPS inputs (chi = 2)
    sample(FockState, U, shots, generator, ...)                        dispatch on the input state
    sample_chains(U, in_modes, sigma, uniforms=...)                     chains with a given column order
    BatchedSampler(circuits, shots, loss=, indist=)                     many circuits, one launch, CUDA graph
    laplace_cofactors_rows(A, rows)                                     the cofactor step alone
    prefix_columns(A, prefix, shots, generator), prefix_columns_many,  column sets for a forced prefix
    prefix_subset_weights(A, prefix)                                    (adaptive sampling)

Mirrors photonic_engines/clifford/__init__.py:36-60 and 139-166 for Fock and EmitterMPS inputs; other
input types (superpositions) are not part of this library and raise.
"""
from __future__ import annotations

import torch

from ..states import EmitterMPS, FockState
from .batch import BatchedSampler
from .emitter import emitter_sample
from .kernels import laplace_cofactors_rows
from .prefix import prefix_columns, prefix_columns_many, prefix_subset_weights
from .sampler import fock_sample, sample_chains

__all__ = ["BatchedSampler", "emitter_sample", "fock_sample", "laplace_cofactors_rows", "prefix_columns",
           "prefix_columns_many", "prefix_subset_weights", "sample", "sample_chains"]


def sample(state, U: torch.Tensor, shots: int, generator: torch.Generator | None = None, **kw):
    """Exact samples [shots, m] for a FockState (`fock_sample` on its modes) or EmitterMPS input
    (`emitter_sample`)."""
    if isinstance(state, FockState):
        return fock_sample(U, state.modes(), shots, generator=generator, **kw)
    if isinstance(state, EmitterMPS):
        return emitter_sample(state, U, shots, generator=generator, **kw)
    raise TypeError(f"unsupported input state {type(state).__name__}: this library samples Fock and EmitterMPS "
                    "inputs only")
