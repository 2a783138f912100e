"""
One process per GPU (torch.distributed) for the two ways the path shards:

* a fit population: independent parameter sets, split across ranks by
  estimated cost (longest first onto the least-loaded rank), evaluated
  locally, curves gathered back in the caller's order;
* one large detector image: q points split into contiguous blocks, every
  rank integrating the same dispersity mesh, the blocks gathered back (the
  four norm sums are identical on every rank, so rank 0's are kept);
* one call with few q and a large mesh: the mesh split into contiguous
  [pd_start, pd_stop) ranges (the restart contract of kernel_iq.c:392-409),
  each rank summing its range from zero, the partial sums gathered and
  added in rank order, so every rank holds the same, reproducible total.

The first two need no reduction on the data path -- the only collective is
the final gather of results, made on device tensors (gather_blocks); the
third has one small exchange (nout*nq + 4 doubles per rank).

Surrogate training runs data-parallel: identical replicas, each global
batch split into equal contiguous slices (`batch_slice`), and one
all-reduce per step of one flat bucket of the ~200k fp32 gradients plus the
loss (`allreduce_mean`), so every replica applies the same Adam update.  The evaluation itself is a callable, the GPU
engine by default, so the host logic here runs (and is tested) with the
gloo backend on CPU as well as NCCL on GPUs.
"""

import numpy as np


def _dist():
    import torch.distributed as dist
    return dist


def world():
    dist = _dist()
    if dist.is_available() and dist.is_initialized():
        return dist.get_world_size(), dist.get_rank()
    return 1, 0


def shard_by_cost(costs, nranks):
    """Assignment of items to ranks: longest-processing-time-first onto the
    least loaded rank.  Deterministic; returns a list of index lists, each in
    increasing order."""
    costs = np.asarray(costs, dtype=float)
    order = np.argsort(-costs, kind="stable")
    load = np.zeros(nranks)
    parts = [[] for _ in range(nranks)]
    for i in order:
        r = int(np.argmin(load))
        parts[r].append(int(i))
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def population_cost(model, sets):
    """Relative cost of each (q, pars) set: q points x mesh points x Gauss
    rule length at the distribution centres."""
    from .batch import _rmax, rule_points
    from .core import load_model_info
    from .direct_model import make_call_args
    info = load_model_info(model)
    costs = []
    for q, pars in sets:
        q = np.asarray(q, 'd')
        details, _, _ = make_call_args(info, pars, [q])
        rmax = _rmax(model, pars, info)
        pts = rule_points(q*rmax) if rmax > 0 else np.ones(q.size)
        costs.append(float(details.num_eval*pts.sum()))
    return costs


def _collective_device():
    """Device the process group's collectives take tensors on: this rank's
    CUDA device for NCCL, the host for gloo."""
    import torch
    dist = _dist()
    if dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def gather_blocks(block, group=None):
    """All-gather one 1D float64 tensor per rank, of lengths that may differ
    between ranks, into their concatenation in rank order on every rank.

    Two collectives on device tensors (no host pickling): the lengths (one
    int64 per rank), then the blocks padded to the longest.  Returns a tensor
    on the collective device."""
    import torch
    dist = _dist()
    size, _ = world()
    dev = _collective_device() if size > 1 else block.device
    block = block.reshape(-1).to(dev, torch.float64)
    if size == 1:
        return block
    n = torch.tensor([block.numel()], dtype=torch.int64, device=dev)
    counts = [torch.empty_like(n) for _ in range(size)]
    dist.all_gather(counts, n, group=group)
    counts = [int(c.item()) for c in counts]
    width = max(max(counts), 1)
    padded = torch.zeros(width, dtype=torch.float64, device=dev)
    padded[:block.numel()] = block
    bufs = [torch.empty_like(padded) for _ in range(size)]
    dist.all_gather(bufs, padded, group=group)
    return torch.cat([b[:c] for b, c in zip(bufs, counts)])


def gather_in_order(local, indices, total):
    """All-gather per-item result arrays (1D, any lengths); returns the full
    list in item order on every rank, as numpy arrays.  The arrays travel as
    one flat device tensor per rank with a small table of item indices and
    lengths (gather_blocks), not as pickled host objects."""
    import torch
    size, _ = world()
    if size == 1:
        out = [None]*total
        for i, v in zip(indices, local):
            out[i] = np.asarray(v.cpu() if isinstance(v, torch.Tensor) else v)
        return out
    dev = _collective_device()
    arrays = [torch.as_tensor(v, dtype=torch.float64).reshape(-1).to(dev) for v in local]
    flat = torch.cat(arrays) if arrays else torch.zeros(0, dtype=torch.float64, device=dev)
    table = torch.tensor([x for i, a in zip(indices, arrays) for x in (i, a.numel())],
                         dtype=torch.float64, device=dev)
    all_table = gather_blocks(table).cpu().numpy().astype(np.int64).reshape(-1, 2)
    all_flat = gather_blocks(flat).cpu().numpy()
    out = [None]*total
    off = 0
    for i, n in all_table:
        out[int(i)] = all_flat[off:off + n]
        off += n
    return out


def evaluate_population(model, sets, evaluate=None, costs=None, **kwargs):
    """I(q) of every set of a population, sharded over the process group.

    *evaluate(model, subset)* returns the list of I(q) arrays of a subset;
    by default the batched GPU engine on this rank's device."""
    size, rank = world()
    if costs is None:
        costs = population_cost(model, sets)
    parts = shard_by_cost(costs, size)
    mine = parts[rank]
    if evaluate is None:
        evaluate = _evaluate_batched
    local = evaluate(model, [sets[i] for i in mine], **kwargs) if mine else []
    return gather_in_order(local, mine, len(sets))


def _evaluate_batched(model, subset, form="float32c", device=None):
    from .batch import Population
    pop = Population(model, subset, form=form, device=device)
    pop.run()
    return pop.iq()


def q_blocks(nq, nranks):
    """Contiguous [lo, hi) q ranges, one per rank."""
    b = np.linspace(0, nq, nranks + 1).astype(int)
    return [(int(b[r]), int(b[r + 1])) for r in range(nranks)]


def evaluate_image(q_vectors, evaluate, nout=1):
    """One image split by q blocks: *evaluate(q_block_vectors)* returns the
    raw result of its block (nout*nq_block slots, then the 4 norms; a numpy
    array or torch tensor); returns the full raw vector (q slots in caller
    order, norms of rank 0) on every rank as a numpy array.  *nout* is 2 for
    1D models returning <F> and <F^2>, else 1: it comes from the model, not
    from the block, so a rank with an empty block (nq < ranks) still
    assembles the image right.  The blocks travel as device tensors
    (gather_blocks)."""
    import torch
    size, rank = world()
    nq = len(q_vectors[0])
    lo, hi = q_blocks(nq, size)[rank]
    raw = evaluate([np.asarray(v)[lo:hi] for v in q_vectors])
    raw = torch.as_tensor(raw, dtype=torch.float64).reshape(-1)
    # every rank takes both collectives, a malformed block included, and
    # only then reports it, so the other ranks are not left waiting
    slots = gather_blocks(raw[:nout*(hi - lo)])
    norms = gather_blocks(raw[nout*(hi - lo):])[:4]      # rank 0's four norms
    if raw.numel() != nout*(hi - lo) + 4:
        raise ValueError("block result has %d values, expected %d"
                         % (raw.numel(), nout*(hi - lo) + 4))
    return torch.cat([slots, norms]).cpu().numpy()


def mesh_ranges(num_eval, nranks):
    """Contiguous [pd_start, pd_stop) mesh ranges, one per rank."""
    b = np.linspace(0, num_eval, nranks + 1).astype(int)
    return [(int(b[r]), int(b[r + 1])) for r in range(nranks)]


def evaluate_mesh(num_eval, evaluate):
    """One call's mesh split over the process group: *evaluate(pd_start,
    pd_stop)* returns the raw sums (F^2 [and F] slots, then the four norms)
    of that mesh range started from zero, as a numpy array or torch tensor;
    the ranks' partial sums are all-gathered and added in rank order, which
    gives every rank the same total whatever the reduction hardware."""
    import torch
    size, rank = world()
    lo, hi = mesh_ranges(num_eval, size)[rank]
    part = evaluate(lo, hi)
    if size == 1:
        return part
    dist = _dist()
    as_numpy = not isinstance(part, torch.Tensor)
    t = torch.as_tensor(np.asarray(part)) if as_numpy else part.contiguous()
    bufs = [torch.empty_like(t) for _ in range(size)]
    dist.all_gather(bufs, t)
    total = bufs[0].clone()
    for b in bufs[1:]:
        total += b
    return total.numpy() if as_numpy else total


def kernel_mesh_partition(kernel, call_details, values, cutoff=0.0, magnetic=False,
                          radius_effective_mode=0):
    """Raw result of one B200Kernel call (the layout of ``kernel.result``,
    in the caller's q order) with its mesh split over the process group,
    one rank per GPU; every rank returns the same summed vector."""
    import torch
    variant = kernel.variant(magnetic)
    dev_d, dev_v = kernel.upload(call_details, values)

    def run(lo, hi):
        with torch.cuda.device(kernel.device), torch.cuda.stream(kernel.stream):
            out = torch.zeros_like(kernel._result_dev)
            if hi > lo:
                kernel.launch(variant, dev_d, dev_v, lo, hi, cutoff, radius_effective_mode,
                              result_dev=out)
        kernel.stream.synchronize()
        return out

    total = evaluate_mesh(call_details.num_eval, run).cpu().numpy()
    raw = total.copy()
    order = kernel.q_input.order
    if order is not None:
        nq = kernel.q_input.nq
        raw[order] = total[:nq]
    return raw


def batch_slice(start, batch, rank, nranks):
    """[lo, hi) of this rank's contiguous slice of the global batch
    [start, start + batch); the slices are equal and cover the batch."""
    if batch % nranks:
        raise ValueError("global batch %d does not split over %d ranks" % (batch, nranks))
    local = batch//nranks
    return start + rank*local, start + (rank + 1)*local


def allreduce_mean(tensors, group=None):
    """Average a list of fp32 tensors in place over the ranks of `group` with
    ONE all-reduce of one flat bucket (the surrogate's gradients and loss).
    Every rank receives the same reduced bits, so replicas that start equal
    stay equal without a parameter broadcast.  Returns the list."""
    import torch
    dist = _dist()
    if not (dist.is_available() and dist.is_initialized()):
        return tensors
    size = dist.get_world_size(group)
    if size == 1:
        return tensors
    flat = torch.cat([t.reshape(-1) for t in tensors])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    flat.div_(size)
    off = 0
    for t in tensors:
        k = t.numel()
        t.view(-1).copy_(flat[off:off + k])
        off += k
    return tensors


def broadcast_parameters(net, src=0, group=None):
    """Copy the surrogate network's fp32 parameters from rank `src` to every
    rank (and refresh its bf16 copies), so data-parallel replicas start from
    the same weights whatever their seeds; optimiser moments stay zero."""
    dist = _dist()
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size(group) == 1:
        return net
    for p in net.params:
        dist.broadcast(p, src, group=group)
    net._sync_bf16()
    return net
