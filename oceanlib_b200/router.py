"""Sharding sea states across GPUs: one process per GPU, no data exchange.

Every ocean, cascade level, ensemble member and session is independent (a
pure function of its seed, descriptor and time), so several GPUs share a
workload by owning disjoint sets of oceans. The only question is which rank
owns which ocean. `assign` answers it the same way on every rank, from the
descriptors alone, so no rank has to tell another anything:

* an ocean's cost is its frame's memory traffic, N^2 x (6 fields with
  velocity, 4 without) - the frame kernels are bound by moving those;
* oceans go, largest cost first (ties by index), to the rank with the least
  cost so far (ties to the lower rank) - the longest-processing-time rule,
  whose largest load exceeds the mean by less than one ocean's cost.

`ShardedEnsemble` builds this rank's share as one OceanEnsemble on its GPU.
"""
from __future__ import annotations

from typing import List, Sequence


def ocean_cost(desc) -> float:
    """Relative frame cost of one ocean: cells x complex fields."""
    return float(desc.size) * float(desc.size) * (6.0 if desc.compute_velocity else 4.0)


def assign(descs: Sequence, world: int) -> List[List[int]]:
    """Indices of `descs` owned by each of `world` ranks (deterministic)."""
    if world < 1:
        raise ValueError("world must be at least 1")
    order = sorted(range(len(descs)), key=lambda i: (-ocean_cost(descs[i]), i))
    load = [0.0] * world
    owned: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owned[r].append(i)
        load[r] += ocean_cost(descs[i])
    return [sorted(o) for o in owned]


def loads(descs: Sequence, shares: List[List[int]]) -> List[float]:
    return [sum(ocean_cost(descs[i]) for i in s) for s in shares]


class ShardedEnsemble:
    """This rank's share of `descs` as one OceanEnsemble on the current GPU.
    `indices` maps the local ensemble's oceans back to positions in `descs`."""

    def __init__(self, descs: Sequence, rank: int, world: int, autotune: bool = True):
        from . import OceanEnsemble

        self.indices = assign(descs, world)[rank]
        self.ensemble = OceanEnsemble([descs[i] for i in self.indices], autotune=autotune) if self.indices else None

    def update(self, time: float, stream: int = 0) -> None:
        if self.ensemble is not None:
            self.ensemble.update(time, stream)

    def synchronize(self) -> None:
        if self.ensemble is not None:
            self.ensemble.synchronize()

    def close(self) -> None:
        if self.ensemble is not None:
            self.ensemble.close()
            self.ensemble = None
