"""Independent fields across the GPUs of a node (one process per GPU).

A field never spans GPUs (its transforms need the whole field; the
reference's MPI slab decomposition, Csource/2dpar main_2d_par.c:139-145 and
fft_routines_2d_par.c, exists to spread one field over CPU ranks).  What
does spread is a set of independent fields -- an ensemble or a stream of
requests: each rank takes a share, advances it on its own GPU with no
collective on the data path, and the results are gathered on the host.

The shares balance the estimated work of a field, n^2 * steps * T_M with
T_M = 6 + M + M(M+1)/2 the 2-D transforms of one right-hand side at order M:
fields are dealt largest first to the rank with the least work so far
(longest-processing-time order), ties by field index, so every rank computes
the same assignment without communicating.
"""
from __future__ import annotations

import heapq


def transforms_per_rhs(order):
    """2-D transforms of one RHS evaluation at HOS order M: 5 + M(M+1)/2
    inverse (eta, its x and y derivatives, the x and y derivatives of phi,
    and the z-derivatives of every phi^(i)) and M + 1 forward."""
    return 6 + order + order * (order + 1) // 2


def work(n, order, steps, ny=None):
    """Estimated work of one field: grid points x steps x transforms per RHS."""
    return float(n) * float(ny if ny is not None else n) * float(steps) * transforms_per_rhs(order)


def assign(works, world):
    """Rank of every item: largest work first, each to the rank with the
    least work so far (lowest rank on ties).  Returns (ranks, load per rank)."""
    order = sorted(range(len(works)), key=lambda i: (-works[i], i))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    ranks = [0] * len(works)
    load = [0.0] * world
    for i in order:
        w, r = heapq.heappop(heap)
        ranks[i] = r
        load[r] = w + works[i]
        heapq.heappush(heap, (load[r], r))
    return ranks, load


class Partition:
    """This rank's share of a list of field specs.

    ``specs`` are any objects; ``work_of(spec)`` gives each one's estimated
    work.  ``mine`` lists (index, spec) of the specs this rank advances;
    ``gather(results)`` (results in the order of ``mine``) returns, on every
    rank, the list of all results in spec order -- the only communication,
    on the host (``torch.distributed.all_gather_object``) after the work.
    With one rank it is the identity."""

    def __init__(self, specs, work_of, rank=0, world=1):
        self.specs = list(specs)
        self.rank, self.world = int(rank), int(world)
        self.ranks, self.load = assign([work_of(s) for s in self.specs], self.world)
        self.mine = [(i, s) for i, s in enumerate(self.specs) if self.ranks[i] == self.rank]

    def imbalance(self):
        """Largest rank's work over the mean (1.0 = perfect balance)."""
        mean = sum(self.load) / max(1, self.world)
        return max(self.load) / mean if mean > 0 else 1.0

    def gather(self, results):
        if len(results) != len(self.mine):
            raise ValueError("one result per spec of this rank")
        mine = [(i, r) for (i, _), r in zip(self.mine, results)]
        if self.world == 1:
            parts = [mine]
        else:
            import torch.distributed as tdist

            parts = [None] * self.world
            tdist.all_gather_object(parts, mine)
        out = [None] * len(self.specs)
        for part in parts:
            for i, r in part:
                out[i] = r
        return out
