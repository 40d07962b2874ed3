"""Input state accepted by the Fock sampler: one n-photon Fock state over m modes
(the reference's `FockState`, photonic_engines/states.py:45-77)."""
from __future__ import annotations

import math
from collections.abc import Sequence
from dataclasses import dataclass


def modes_from_occupation(occ: Sequence[int]) -> list[int]:
    """Occupation [s_1 .. s_m] -> input modes with multiplicity, ascending."""
    return [j for j, c in enumerate(occ) for _ in range(int(c))]


@dataclass(frozen=True)
class FockState:
    """|s_1 ... s_m>: `occupation` is the photon count per mode (non-negative ints, at least one mode)."""

    occupation: tuple[int, ...]

    def __post_init__(self):
        occ = tuple(int(x) for x in self.occupation)
        if any(x < 0 for x in occ) or not occ:
            raise ValueError("occupation must be a non-empty tuple of non-negative ints")
        object.__setattr__(self, "occupation", occ)

    @property
    def n(self) -> int:
        return sum(self.occupation)

    @property
    def m(self) -> int:
        return len(self.occupation)

    def modes(self) -> list[int]:
        """Input modes with multiplicity (the columns of U the sampler uses)."""
        return modes_from_occupation(self.occupation)

    def norm_factor(self) -> float:
        return math.prod(math.factorial(x) for x in self.occupation)
