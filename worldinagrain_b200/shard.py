"""Worlds across GPUs: a batch's worlds are independent, so N ranks (one
process per GPU) each step their own share with no collective on the data
path; only the host-side bookkeeping (which rank owns which world, the
timing's max over ranks, the latencies for the percentiles) crosses ranks.
A single world does not shard (every smoother sweep needs its neighbours
and every CG iteration two global sums): it runs as replicas.

The share is a greedy bin-pack by cells: worlds largest first, each to the
rank with the fewest cells so far (ties to the lowest rank), so every rank
ends within one world's cells of the others.
"""
import heapq


def partition(cells, n_ranks):
    """Worlds (their cell counts) into n_ranks shares of about equal cells:
    a list of n_ranks sorted lists of world indices."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be at least 1")
    order = sorted(range(len(cells)), key=lambda k: (-cells[k], k))
    heap = [(0, r) for r in range(n_ranks)]
    shares = [[] for _ in range(n_ranks)]
    for k in order:
        load, r = heapq.heappop(heap)
        shares[r].append(k)
        heapq.heappush(heap, (load + cells[k], r))
    return [sorted(s) for s in shares]


def share_of(cells, rank, n_ranks):
    """This rank's worlds."""
    return partition(cells, n_ranks)[rank]


def route(world, owner):
    """The rank that serves a request for `world` (owner: world -> rank)."""
    return owner[world]


def owners(shares):
    """world -> rank, from partition()'s shares."""
    out = {}
    for r, s in enumerate(shares):
        for k in s:
            out[k] = r
    return out
