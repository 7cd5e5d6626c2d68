"""Right-hand-side replicas across GPUs (one process per GPU).

Every rank holds a full replica of the tree, lists and operators and
evaluates its own contiguous block of the k right-hand sides; no data moves
between GPUs during an evaluate.  The helpers here are the host-side plumbing
around that: the block of right-hand sides a rank owns, the all-gather that
assembles every rank's values when a caller wants them everywhere, and the
max-over-ranks reduction of a step time (the slowest rank sets the job's time).
They take any torch.distributed process group (NCCL on GPUs, gloo on CPU).
"""
import torch
import torch.distributed as dist


def rhs_block(k_total, world, rank):
    """(first, count) of the contiguous block of right-hand sides rank owns;
    the first k_total % world ranks take one extra."""
    if k_total < 0 or world < 1 or not 0 <= rank < world:
        raise ValueError("bad k_total/world/rank")
    base, extra = divmod(k_total, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def evaluate_replicated(evaluate_block, dens, group=None):
    """Evaluate dens ([k_total, n_src*srcDOF], the same on every rank) as
    right-hand-side replicas: this rank runs evaluate_block on its own block
    (a [count, ...] tensor in, a [count, n_trg*trgDOF] tensor out) and the
    blocks are all-gathered, so every rank returns the [k_total, ...] values.
    evaluate_block is called on every rank, possibly with an empty block."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    k_total = dens.shape[0]
    first, count = rhs_block(k_total, world, rank)
    local = evaluate_block(dens[first:first + count])
    width = local.shape[1] if local.dim() == 2 else 0
    sizes = [rhs_block(k_total, world, r)[1] for r in range(world)]
    widths = [torch.zeros(1, dtype=torch.int64, device=local.device) for _ in range(world)]
    dist.all_gather(widths, torch.tensor([width], dtype=torch.int64, device=local.device), group=group)
    width = max(int(w.item()) for w in widths)
    pad = max(sizes)
    buf = torch.zeros((pad, width), dtype=local.dtype, device=local.device)
    if count:
        buf[:count] = local
    parts = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    return torch.cat([parts[r][:sizes[r]] for r in range(world)], dim=0)


def max_over_ranks(value, device=None, group=None):
    """The largest of every rank's value (a step time in ms)."""
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
