"""Temperature replica exchange of one ladder split over ranks (one process
per GPU), the layout the reference uses with MPI: each rank owns a
contiguous block of the replicas, computes replica_energy(2, ·) of its own
(energy_allrep.F90:123-217), the ranks gather those arrays in replica order
(time_integral_post.F90:279), and every rank then applies the same exchange
(simu_replica_exchange.F90:121-267) to the whole ladder's label maps,
relabelling and rescaling only its own replicas.  No coordinates move
between ranks; the only collective is the all-gather of 2 doubles per
replica at each exchange.
"""
from __future__ import annotations

import numpy as np


def ladder_share(nrep_all: int, world: int, rank: int) -> tuple[int, int]:
    """(first replica, 1-based; count) of rank's block: contiguous, sizes
    differing by at most one, lower ranks taking the larger blocks."""
    if not (0 <= rank < world) or nrep_all < world:
        raise ValueError("every rank needs at least one replica")
    base, extra = divmod(nrep_all, world)
    count = base + (1 if rank < extra else 0)
    first = rank * base + min(rank, extra) + 1
    return first, count


def gather_energies(local: np.ndarray, nrep_all: int, dist=None, device: str = "cpu") -> np.ndarray:
    """(nrep_all, 2) replica energies in replica order from every rank's
    (count, 2) block (torch.distributed all_gather; blocks padded to the
    largest)."""
    local = np.asarray(local, dtype=np.float64).reshape(-1, 2)
    if dist is None:
        assert local.shape[0] == nrep_all
        return local.copy()
    import torch
    world = dist.get_world_size()
    width = -(-nrep_all // world)
    buf = torch.zeros((width, 2), dtype=torch.float64, device=device)
    buf[:local.shape[0]] = torch.from_numpy(local).to(device)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    out = []
    for r, t in enumerate(parts):
        _, count = ladder_share(nrep_all, world, r)
        out.append(t[:count].cpu().numpy())
    return np.concatenate(out)


class LadderExchange:
    """Exchanges for a ladder engine (Engine(..., ladder=(tempk_all, first)))
    over a torch.distributed group (None: a single process)."""

    def __init__(self, engine, nrep_all: int, dist=None, device: str = "cpu"):
        self.engine = engine
        self.nrep_all = nrep_all
        self.dist = dist
        self.device = device

    def exchange(self, u=None) -> int:
        e = gather_energies(self.engine.rex_energies(), self.nrep_all, self.dist, self.device)
        return self.engine.rex_exchange_all(e, u)
