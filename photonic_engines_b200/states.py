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


@dataclass(frozen=True)
class EmitterMPS:
    """Photons emitted one by one by a single emitter of dimension chi (the reference's `EmitterMPS`,
    photonic_engines/states.py:306-420): at event k the emitter emits label l into input mode modes[k][l]
    and is acted on by ops[k, l]; the photonic amplitude of labels x is <final| ops[n-1, x_{n-1}] ...
    ops[0, x_0] |s0>, or the emitter is traced out when `final` is None.

    ops [n, L, chi, chi] complex; modes: n tuples of L_k <= L distinct input modes (all distinct across
    events); s0 [chi]; m >= 1 + max mode; final [chi] or None.  Padded labels (l >= L_k) must have zero
    operators."""

    ops: object
    modes: tuple
    s0: object
    m: int
    final: object = None

    def __post_init__(self):
        import numpy as np
        ops = np.asarray(self.ops, dtype=np.complex128)
        if ops.ndim != 4 or ops.shape[2] != ops.shape[3]:
            raise ValueError("ops must have shape [n, L, chi, chi]")
        n, L, chi, _ = ops.shape
        modes = tuple(tuple(int(x) for x in mk) for mk in self.modes)
        if len(modes) != n or any(not 1 <= len(mk) <= L for mk in modes):
            raise ValueError("modes must have shape [n][L_k] with 1 <= L_k <= L")
        for k, mk in enumerate(modes):
            if np.any(ops[k, len(mk):]):
                raise ValueError(f"ops[{k}, {len(mk)}:] must be zero: event {k} has {len(mk)} labels")
        flat = [x for mk in modes for x in mk]
        if len(set(flat)) != len(flat):
            raise ValueError("every (event, label) must use a distinct input mode")
        if min(flat) < 0 or max(flat) >= int(self.m):
            raise ValueError("mode index out of range")
        s0 = np.asarray(self.s0, dtype=np.complex128).reshape(-1)
        if s0.shape != (chi,):
            raise ValueError("s0 must have length chi")
        final = None if self.final is None else np.asarray(self.final, dtype=np.complex128).reshape(-1)
        if final is not None and final.shape != (chi,):
            raise ValueError("final must have length chi")
        object.__setattr__(self, "ops", ops)
        object.__setattr__(self, "modes", modes)
        object.__setattr__(self, "s0", s0)
        object.__setattr__(self, "final", final)
        object.__setattr__(self, "m", int(self.m))

    @property
    def n(self) -> int:
        return self.ops.shape[0]

    @property
    def num_labels(self) -> int:
        return self.ops.shape[1]

    @property
    def chi(self) -> int:
        return self.ops.shape[2]

    @property
    def is_ragged(self) -> bool:
        return any(len(mk) < self.num_labels for mk in self.modes)

    def require_uniform_labels(self, where: str):
        """NotImplementedError for a chain whose events have different label counts."""
        if self.is_ragged:
            raise NotImplementedError(f"ragged label counts ({tuple(len(mk) for mk in self.modes)}): not in {where}")


def spin_gate(theta: float, phi: float):
    """Ry(theta/2) Rz(phi) Ry(theta/2) (2 x 2): the spin rotation between two emissions of a caterpillar
    emitter (the reference's `spin_gate`, photonic_engines/states.py:850-861)."""
    import numpy as np

    def ry(t):
        c, s = math.cos(t / 2), math.sin(t / 2)
        return np.array([[c, -s], [s, c]], dtype=np.complex128)

    rz = np.diag([np.exp(-0.5j * phi), np.exp(0.5j * phi)]).astype(np.complex128)
    return ry(theta / 2) @ rz @ ry(theta / 2)


def caterpillar(n: int, spin_gates, m: int | None = None, modes=None, s0=(1.0, 0.0), final=None) -> EmitterMPS:
    """A spin emitting photon k into mode modes[k][0] when up and modes[k][1] when down, after the spin gate
    spin_gates[k] (the reference's `EmitterMPS.caterpillar`, photonic_engines/states.py:455-483): ops[k, 0] =
    P_up G_k, ops[k, 1] = P_down G_k; default modes (2k, 2k + 1) and m = 2n.  spin_gate(pi/2, 0) everywhere
    gives the linear cluster state."""
    import numpy as np
    if len(spin_gates) != n:
        raise ValueError("one spin gate per emission")
    modes = [(2 * k, 2 * k + 1) for k in range(n)] if modes is None else modes
    m = max(x for mk in modes for x in mk) + 1 if m is None else m
    up, down = np.diag([1.0, 0.0]).astype(np.complex128), np.diag([0.0, 1.0]).astype(np.complex128)
    ops = np.stack([np.stack([up @ np.asarray(G, dtype=np.complex128), down @ np.asarray(G, dtype=np.complex128)])
                    for G in spin_gates])
    return EmitterMPS(ops=ops, modes=tuple(tuple(mk) for mk in modes), s0=s0, m=m, final=final)
