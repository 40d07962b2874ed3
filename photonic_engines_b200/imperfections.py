"""Input-side photon loss and partial distinguishability for the Fock sampler (host logic).

Model (the reference's shared imperfections model, photonic_engines/imperfections.py:1-60, 465-590):
every input photon is lost with probability 1 - eta; a surviving photon draws a species — in the
x-model it interferes with probability x and is otherwise alone in an orthogonal internal mode
(a "singleton"); with `species` probabilities q_mu it joins species mu, and the remainder makes it a
singleton.  Photons of one species form an ordinary lossless instance on their columns; a singleton
lands in row r with probability |U[r, col]|^2.

The draws here consume the generator with the same torch calls, in the same order, as the reference
(`draw_roles` :529-548, `partition` :551-573, `route_classical` :576-590), so that a seeded
generator gives the same partition of the shots.  This is host bookkeeping: the chains of every
partition run in one launch of the CUDA chain kernel.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import torch

LOST, SINGLE = 0, 1          # roles; interfering species mu has role 2 + mu


def _eta(eta):
    """None or a transmission >= 1 means no loss; otherwise the transmission, checked to lie in [0, 1]."""
    if eta is None:
        return None
    if isinstance(eta, torch.Tensor):
        return None if float(eta.detach()) >= 1.0 else eta
    e = float(eta)
    if not 0.0 <= e <= 1.0:
        raise ValueError(f"loss (transmission) must be in [0, 1], got {e}")
    return None if e >= 1.0 else e


@dataclass(frozen=True)
class Distinguishability:
    """x-model (`x`: pairwise overlap, V_HOM = x^2) or random species (`species`: probabilities q_mu of the
    interfering species, sum <= 1, the remainder being a photon alone in its own mode)."""
    x: float | None = None
    species: tuple[float, ...] | None = None

    def __post_init__(self):
        if (self.x is None) == (self.species is None):
            raise ValueError("give exactly one of x (x-model) or species (random species probabilities)")
        if self.x is not None:
            if not 0.0 <= float(self.x) <= 1.0:
                raise ValueError(f"x must be in [0, 1], got {self.x}")
            object.__setattr__(self, "x", float(self.x))
        else:
            q = tuple(float(v) for v in self.species)
            if any(v < 0 for v in q) or sum(q) > 1.0 + 1e-12:
                raise ValueError("species probabilities must be non-negative and sum to at most 1")
            object.__setattr__(self, "species", q)

    @staticmethod
    def from_hom_visibility(V: float) -> "Distinguishability":
        if not 0.0 <= float(V) <= 1.0:
            raise ValueError(f"visibility must be in [0, 1], got {V}")
        return Distinguishability(x=math.sqrt(float(V)))

    @property
    def probs(self) -> tuple[float, ...]:
        return (self.x,) if self.x is not None else self.species

    @property
    def is_ideal(self) -> bool:
        return sum(self.probs) >= 1.0 and len([q for q in self.probs if q > 0]) == 1


def spec(indist) -> Distinguishability | None:
    """Normalise `indist=`: None / 1.0 / an ideal spec -> None (the lossless path); a float is the x-model; a
    sequence of per-photon overlaps is checked and reduced to the x-model of its smallest overlap."""
    if indist is None:
        return None
    if isinstance(indist, (list, tuple)) or (isinstance(indist, torch.Tensor) and indist.dim() == 1):
        xs = [float(v) for v in indist]
        if any(not 0.0 <= v <= 1.0 for v in xs):
            raise ValueError("per-photon overlaps must be in [0, 1]")
        return None if all(v >= 1.0 for v in xs) else Distinguishability(x=min(xs))
    d = indist if isinstance(indist, Distinguishability) else Distinguishability(
        x=float(indist.detach()) if isinstance(indist, torch.Tensor) else float(indist))
    return None if d.is_ideal else d


def draw_roles(n: int, shots: int, eta, indist, generator: torch.Generator | None = None) -> torch.Tensor:
    """Roles [shots, n] (CPU int64): LOST, SINGLE or 2 + species of every input photon of every shot."""
    if generator is None:
        generator = torch.Generator().manual_seed(0)
    e = _eta(eta)
    d = spec(indist)
    roles = torch.full((shots, n), 2, dtype=torch.long)
    if n == 0:
        return roles
    if d is not None:
        q = torch.tensor([*d.probs, max(0.0, 1.0 - sum(d.probs))], dtype=torch.float64)
        mu = torch.multinomial(q, shots * n, replacement=True, generator=generator).view(shots, n)
        roles = torch.where(mu == len(d.probs), torch.full_like(mu, SINGLE), mu + 2)
    if e is not None:
        lost = torch.rand((shots, n), generator=generator) >= float(e)
        roles[lost] = LOST
    return roles


def partition(n: int, shots: int, eta, indist, generator: torch.Generator | None = None, streams=None):
    """Shots grouped by identical role rows: [(species_subsets, singles, stream_ids)], groups in the order of
    torch.unique over the role rows, stream ids (CPU int64) in stable order within a group."""
    ids = torch.arange(shots) if streams is None else torch.as_tensor(streams).reshape(-1).cpu()
    roles = draw_roles(n, shots, eta, indist, generator)
    uniq, inv = torch.unique(roles, dim=0, return_inverse=True)
    order = torch.argsort(inv, stable=True)
    counts = torch.bincount(inv, minlength=uniq.shape[0])
    groups, start = [], 0
    for g, c in enumerate(counts.tolist()):
        row = uniq[g].tolist()
        n_species = max([r - 2 for r in row if r >= 2] + [-1]) + 1
        subsets = tuple(s for s in (tuple(j for j in range(n) if row[j] == 2 + mu) for mu in range(n_species)) if s)
        singles = tuple(j for j in range(n) if row[j] == SINGLE)
        groups.append((subsets, singles, ids[order[start:start + c]]))
        start += c
    return groups


def route_classical(U: torch.Tensor, circuit, cols, generator: torch.Generator | None = None) -> torch.Tensor:
    """Output rows [P] of P photons that interfere with nothing: photon p enters column cols[p] of circuit
    U[circuit[p]] and lands in row r with probability |U[r, col]|^2 (drawn on the host)."""
    if U.dim() == 2:
        U = U[None]
    cols = torch.as_tensor(cols, dtype=torch.long)
    circuit = torch.as_tensor(circuit, dtype=torch.long)
    if cols.numel() == 0:
        return torch.zeros(0, dtype=torch.long)
    p = (U[circuit.to(U.device), :, cols.to(U.device)].abs() ** 2).to("cpu", torch.float64)
    p = p / p.sum(1, keepdim=True)
    return torch.multinomial(p, 1, generator=generator)[:, 0]
