"""Photon loss and partial distinguishability at the input of the Fock sampler: the model, and the host
draws that split the shots of a call into independent chains.

Model.  Every input photon survives with probability eta (the transmission).  A survivor then draws its
internal state: it joins interfering species mu with probability w_mu, or, with the remaining probability
1 - sum(w), it is alone in an internal mode of its own (a "lone" photon).  The x-model is the one-species
case w = (x,), x the pairwise overlap (HOM visibility x^2).  Photons of one species interfere as an
ordinary lossless Fock input on their columns; a lone photon leaves through row r with probability
|U[r, col]|^2.  This is the reference's shared imperfections model (photonic_engines/imperfections.py).

Draws.  A seeded generator must give the reference's samples, so four things follow the reference's use of
the generator (photonic_engines/imperfections.py:529-590) and nothing else does:
  1. one `torch.multinomial` over (w_0, w_1, ..., 1 - sum w), shots * n draws with replacement, read as
     [shots, n] row-major (only when the photons are not all alike);
  2. then one `torch.rand((shots, n))` whose entries >= eta mark lost photons (only under loss);
  3. the shots grouped by their row of fates in lexicographic order of the codes lost < lone < species 0
     < species 1 < ..., the shots of a group in ascending order;
  4. the lone photons routed last, by one `torch.multinomial` over the rows |U[:, col]|^2 (float64, each
     row divided by its sum), one draw per photon.
"""
from __future__ import annotations

import math
from typing import NamedTuple

import torch

LOST, LONE = -1, 0           # fate codes; interfering species mu is 1 + mu (the order the grouping uses)


class Distinguishability:
    """Partial distinguishability of the input photons, in one of two parametrisations:

        Distinguishability(x=0.95)              the x-model: each photon interferes with probability x
        Distinguishability(species=(0.6, 0.3))  probabilities of the interfering species, the rest lone
        Distinguishability.from_hom_visibility(V)   the x-model with x = sqrt(V)
    """

    __slots__ = ("x", "species")

    def __init__(self, x: float | None = None, species=None):
        if (x is None) == (species is None):
            raise ValueError("Distinguishability takes either x (x-model overlap) or species (probabilities of "
                             "the interfering species) -- exactly one of them")
        if x is not None:
            x = float(x)
            if not (0.0 <= x <= 1.0):
                raise ValueError(f"the x-model overlap lies in [0, 1]; got {x}")
            object.__setattr__(self, "x", x)
            object.__setattr__(self, "species", None)
        else:
            w = tuple(float(v) for v in species)
            if min(w, default=0.0) < 0.0 or sum(w) > 1.0 + 1e-12:
                raise ValueError(f"species probabilities must be >= 0 with a sum of at most 1; got {w}")
            object.__setattr__(self, "x", None)
            object.__setattr__(self, "species", w)

    def __setattr__(self, name, value):
        raise AttributeError("Distinguishability is immutable")

    @classmethod
    def from_hom_visibility(cls, V: float) -> "Distinguishability":
        """The x-model of a Hong-Ou-Mandel visibility V = x^2."""
        V = float(V)
        if not (0.0 <= V <= 1.0):
            raise ValueError(f"a HOM visibility lies in [0, 1]; got {V}")
        return cls(x=math.sqrt(V))

    @property
    def weights(self) -> tuple[float, ...]:
        """Probabilities of the interfering species (the x-model: one species, weight x)."""
        return (self.x,) if self.species is None else self.species

    @property
    def ideal(self) -> bool:
        """Every photon in one common species for sure: the photons are indistinguishable."""
        w = self.weights
        return sum(w) >= 1.0 and sum(1 for v in w if v > 0.0) == 1

    def __eq__(self, other):
        return isinstance(other, Distinguishability) and (self.x, self.species) == (other.x, other.species)

    def __hash__(self):
        return hash((self.x, self.species))

    def __repr__(self):
        return f"Distinguishability(x={self.x})" if self.species is None else \
            f"Distinguishability(species={self.species})"


def as_model(indist) -> Distinguishability | None:
    """The `indist=` argument as a model, or None when the photons are indistinguishable.  Accepts None, an
    overlap x (float or 0-d tensor, the x-model), a Distinguishability, or one overlap per photon (a
    sequence: the x-model of the smallest one)."""
    if indist is None:
        return None
    if isinstance(indist, Distinguishability):
        model = indist
    elif isinstance(indist, (list, tuple)) or (isinstance(indist, torch.Tensor) and indist.dim() == 1):
        per_photon = [float(v) for v in indist]
        bad = [v for v in per_photon if not (0.0 <= v <= 1.0)]
        if bad:
            raise ValueError(f"per-photon overlaps lie in [0, 1]; got {bad}")
        if min(per_photon, default=1.0) >= 1.0:
            return None
        model = Distinguishability(x=min(per_photon))
    else:
        model = Distinguishability(x=float(indist.detach()) if isinstance(indist, torch.Tensor) else float(indist))
    return None if model.ideal else model


def transmission(eta) -> float | None:
    """The `loss=` argument: a transmission eta in [0, 1]; None or 1 mean no loss."""
    if eta is None:
        return None
    e = float(eta.detach()) if isinstance(eta, torch.Tensor) else float(eta)
    if not (0.0 <= e <= 1.0):
        raise ValueError(f"loss is a transmission in [0, 1]; got {e}")
    return None if e == 1.0 else e


def draw_fates(n: int, shots: int, eta, indist, generator: torch.Generator | None = None) -> torch.Tensor:
    """Fates [shots, n] (CPU int64) of every input photon: LOST, LONE or 1 + species.  Without a generator
    the draws come from a generator seeded with 0 (every call then partitions alike, as the reference's)."""
    gen = generator if generator is not None else torch.Generator().manual_seed(0)
    fates = torch.ones((shots, n), dtype=torch.int64)                 # species 0: interfering
    if n == 0:
        return fates
    model = as_model(indist)
    if model is not None:
        w = model.weights
        probs = torch.tensor([*w, max(0.0, 1.0 - sum(w))], dtype=torch.float64)
        pick = torch.multinomial(probs, shots * n, replacement=True, generator=gen).view(shots, n)
        fates = torch.where(pick == len(w), torch.full_like(pick, LONE), pick + 1)
    e = transmission(eta)
    if e is not None:
        fates = fates.masked_fill(torch.rand((shots, n), generator=gen) >= e, LOST)
    return fates


class FateGroup(NamedTuple):
    """Shots that drew the same fates: one sorted tuple of photon indices per non-empty interfering species
    (in species order), the lone photons, and the shot ids (ascending)."""
    species: tuple[tuple[int, ...], ...]
    lone: tuple[int, ...]
    shots: torch.Tensor


def group_fates(fates: torch.Tensor, shot_ids: torch.Tensor | None = None) -> list[FateGroup]:
    """The shots grouped by identical fate rows, groups in lexicographic order of the rows (the codes order
    lost < lone < species): a stable radix sort over the photons from the last to the first, then a cut
    wherever two consecutive sorted rows differ."""
    S, n = fates.shape
    ids = torch.arange(S) if shot_ids is None else torch.as_tensor(shot_ids).reshape(-1).cpu()
    if S == 0:
        return []
    order = torch.arange(S)
    for j in range(n - 1, -1, -1):                                    # least significant photon first
        order = order[torch.sort(fates[order, j], stable=True).indices]
    srt = fates[order]
    if n:
        new = torch.ones(S, dtype=torch.bool)
        new[1:] = (srt[1:] != srt[:-1]).any(1)
    else:
        new = torch.zeros(S, dtype=torch.bool)
        new[0] = True
    starts = torch.nonzero(new)[:, 0].tolist() + [S]
    groups = []
    for a, b in zip(starts[:-1], starts[1:]):
        members: dict[int, list[int]] = {}
        for j, f in enumerate(srt[a].tolist()):
            members.setdefault(f, []).append(j)
        species = tuple(tuple(members[c]) for c in sorted(members) if c > LONE)
        groups.append(FateGroup(species, tuple(members.get(LONE, ())), ids[order[a:b]]))
    return groups


def route_lone_photons(U: torch.Tensor, circuit, cols, generator: torch.Generator | None = None) -> torch.Tensor:
    """Output rows [P] of P lone photons: photon p enters column cols[p] of circuit U[circuit[p]] (U [B, m, m]
    or [m, m]) and leaves through row r with probability |U[r, col]|^2 (one host draw per photon)."""
    cols = torch.as_tensor(cols, dtype=torch.long)
    if cols.numel() == 0:
        return torch.zeros(0, dtype=torch.long)
    Ub = U if U.dim() == 3 else U.unsqueeze(0)
    dev = Ub.device
    circuit = torch.as_tensor(circuit, dtype=torch.long)
    w = (Ub[circuit.to(dev), :, cols.to(dev)].abs() ** 2).to("cpu", torch.float64)      # [P, m]
    w = w / w.sum(1, keepdim=True)
    return torch.multinomial(w, 1, generator=generator)[:, 0]
