"""One likelihood evaluated across GPUs: one process per GPU, the pair sweep
split by target strips.

Every rank holds a :class:`~hawkes_b200.engine.CudaHawkes` engine with all N
events and the same parameters (the events are O(N): 24 bytes each at D = 2).
An evaluation is

1. ``hphc_sweep_shard``: this rank's target strips (whole strips, the same
   deterministic balance on every rank) into a share of every event's six unit
   pair sums, 6 N doubles;
2. one all-gather of those shares over the process group (NCCL over NVLink on
   GPUs; any backend whose tensors live where the engine reads them);
3. ``hphc_set_unit_sums``: the engine adds the shares in rank order, so every
   rank holds the same bits, and the O(N) finish then gives every rank the same
   log-likelihood, gradient and P_i.

The exchange is 6 N doubles per rank per evaluation (4.8 MB at N = 100,000),
against an O(N^2 / world) sweep.  The reference evaluates on one device only;
this is the multi-GPU form of its ``getSumOfLikContribs`` /
``getProbsSelfExcite`` (src/AbstractHawkes.hpp:42-45).
"""
from __future__ import annotations

from typing import Optional

import numpy as np


class ShardedHawkes:
    """Sharded evaluation on `engine` (this rank's engine) over `group`.

    Without an initialised process group the world is this process alone.
    `device`: where the shares live (default: the engine's CUDA device)."""

    def __init__(self, engine, group=None, device=None):
        import torch
        import torch.distributed as dist
        self._torch = torch
        self.engine = engine
        self.group = group
        self._dist = dist if dist.is_available() and dist.is_initialized() else None
        self.rank = self._dist.get_rank(group) if self._dist else 0
        self.world = self._dist.get_world_size(group) if self._dist else 1
        self.device = torch.device(device) if device is not None else \
            torch.device("cuda", engine.device)
        n = 6 * engine.locationCount
        self._all = torch.empty(self.world * n, dtype=torch.float64, device=self.device)
        self._part = self._all[self.rank * n:(self.rank + 1) * n]
        self._send = torch.empty(n, dtype=torch.float64, device=self.device) \
            if self._dist else None

    def _sync(self) -> None:
        if self.device.type == "cuda":
            self._torch.cuda.current_stream(self.device).synchronize()

    def sweep(self) -> None:
        """Steps 1-3: afterwards this rank's engine holds the full unit sums at
        its current parameters."""
        if self._dist is None:
            self.engine.sweepShard(0, 1, self._part.data_ptr())
            self.engine.setUnitSums(self._all.data_ptr(), 1)
            return
        self.engine.sweepShard(self.rank, self.world, self._send.data_ptr())
        self._dist.all_gather_into_tensor(self._all, self._send, group=self.group)
        self._sync()
        self.engine.setUnitSums(self._all.data_ptr(), self.world)

    def getLogLikelihoodAndGradient(self):
        self.sweep()
        return self.engine.getLogLikelihoodAndGradient()

    def getSumOfLikContribs(self) -> float:
        self.sweep()
        return self.engine.getSumOfLikContribs()

    def getLogLikelihoodGradient(self) -> np.ndarray:
        self.sweep()
        return self.engine.getLogLikelihoodGradient()

    def getProbsSelfExcite(self) -> np.ndarray:
        self.sweep()
        return self.engine.getProbsSelfExcite()

    def shares(self) -> Optional[np.ndarray]:
        """The gathered shares of the last sweep (world x 6 x N), on the host."""
        return self._all.reshape(self.world, 6, -1).cpu().numpy()
