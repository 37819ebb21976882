"""Partition-per-rank merge protocol: the reference's distributed merge
(src/cc_mpi.c:535-742) and halo-exchange plan / delta exchange
(src/exchange_plan.c:48-225, 242-425) with one partition per process, over
torch.distributed (NCCL between GPUs, gloo on CPU).

On one GPU the partitioned solver keeps every partition in HBM and does the
exchange as an in-HBM pass (ccgpu_dist_cc).  With one partition per GPU the
exchange crosses processes; this module is that host-side protocol, the same
collective steps in the same order as the reference:

* plan build: every rank sends each owner the ids of the ghosts it needs
  from it - counts by all_to_all, ids by all_to_all with splits (the
  reference's MPI_Alltoall + MPI_Alltoallv, exchange_plan.c:95-142);
* merge rounds: one local round, then the (pending, changed) flags
  OR-reduced across ranks (all_reduce MAX of two ints, cc_mpi.c:634-635);
  exchange when ``exchange_interval`` rounds have passed or nothing changed
  anywhere; stop after a round in which nothing changed since the last
  exchange;
* delta exchange: each rank packs ``(position << 32) | label`` for every
  vertex a neighbour needs whose label fell below what was last sent to it
  (the ``prev_sent`` rule, exchange_plan.c:325-357), counts go by
  all_to_all, pairs by all_to_all with splits, and the receiver writes them
  into its ghost labels (exchange_plan.c:390-413);
* roots: the per-rank root counts are summed (cc_mpi.c:739).

The per-partition work is an *engine* object; the protocol never touches
labels itself.  An engine provides:

  ``has_work()``            1 when the partition has ghosts, pairs and reps
  ``need_from(world)``      list over owner ranks of the global ids (uint32)
                            of the ghosts it needs from each, in ghost order
  ``set_send_to(lists)``    the ids each rank needs from this partition
  ``round()``               one merge round (INIT, HOOK, UPD); returns 1 if a
                            label fell
  ``pack()``                list over destination ranks of uint64 messages
  ``scatter(src, msgs)``    applies the messages received from rank ``src``
  ``roots()``               vertices of this partition that are their
                            component's minimum

Every rank takes every collective step in the same order, including ranks
whose partition has nothing to exchange, so no rank waits on a collective
another rank skipped.
"""
from __future__ import annotations

import numpy as np


def _a2a_counts(dist, torch, counts, device):
    send = torch.tensor(counts, dtype=torch.int64, device=device)
    recv = torch.empty_like(send)
    dist.all_to_all_single(recv, send)
    return recv.tolist()


def _a2a_payload(dist, torch, chunks, recv_counts, dtype, device):
    """all_to_all with splits of numpy arrays; returns one array per source."""
    send_counts = [len(c) for c in chunks]
    flat = np.concatenate(chunks) if sum(send_counts) else np.zeros(0, dtype=dtype)
    send = torch.from_numpy(flat.view(np.int64) if dtype == np.uint64 else
                            flat.astype(np.int64)).to(device)
    recv = torch.empty(sum(recv_counts), dtype=torch.int64, device=device)
    dist.all_to_all_single(recv, send, output_split_sizes=recv_counts,
                           input_split_sizes=send_counts)
    out = recv.cpu().numpy()
    out = out.view(np.uint64) if dtype == np.uint64 else out.astype(dtype)
    parts, o = [], 0
    for c in recv_counts:
        parts.append(out[o:o + c])
        o += c
    return parts


def _or_max(dist, torch, flags, device):
    t = torch.tensor(flags, dtype=torch.int64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [int(x) for x in t.tolist()]


def build_plan(engine, dist, torch, device="cpu"):
    """exchangeplan_build (src/exchange_plan.c:48-225): returns
    (indegree, outdegree, total_send_to, total_need_from)."""
    world = dist.get_world_size()
    need = engine.need_from(world)
    need_counts = [len(x) for x in need]
    send_counts = _a2a_counts(dist, torch, need_counts, device)
    send_to = _a2a_payload(dist, torch, [np.asarray(x, np.int64) for x in need], send_counts,
                           np.uint32, device)
    engine.set_send_to(send_to)
    return (sum(1 for c in need_counts if c), sum(1 for c in send_counts if c),
            sum(send_counts), sum(need_counts))


def exchange(engine, dist, torch, device="cpu"):
    """exchangeplan_exchange_delta (src/exchange_plan.c:242-425); returns the
    pairs this rank sent."""
    msgs = engine.pack()
    counts = _a2a_counts(dist, torch, [len(x) for x in msgs], device)
    recv = _a2a_payload(dist, torch, msgs, counts, np.uint64, device)
    for src, m in enumerate(recv):
        if len(m):
            engine.scatter(src, m)
    return sum(len(x) for x in msgs)


def merge(engine, dist, torch, exchange_interval=1, device="cpu"):
    """The merge loop and its exchange schedule (src/cc_mpi.c:535-742).
    Returns a dict with rounds, exchanges, sent pairs (this rank) and the
    global component count."""
    interval = max(1, int(exchange_interval))
    build_plan(engine, dist, torch, device)
    global_pending = _or_max(dist, torch, [int(engine.has_work())], device)[0]
    pending = global_pending
    rounds = exchanges = sent = steps = 0
    while global_pending:
        changed = int(engine.round())
        if changed:
            pending = 1
        global_pending, any_changed = _or_max(dist, torch, [pending, changed], device)
        rounds += 1
        if not global_pending:
            break
        steps += 1
        if steps >= interval or not any_changed:
            sent += exchange(engine, dist, torch, device)
            exchanges += 1
            pending = 0
            steps = 0
    t = torch.tensor([int(engine.roots())], dtype=torch.int64, device=device)
    dist.all_reduce(t)
    return {"rounds": rounds, "exchanges": exchanges, "sent_pairs": sent,
            "components": int(t.item())}
