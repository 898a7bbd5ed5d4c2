"""One MSWS sketch sharded by bucket across the ranks of a process group.

A key's whole state is one low bucket and the high bucket it may link to (reference
device_sketch_v3.h:228, :119, :185), so the sketch partitions by bucket with no state shared
between shards.  Bucket b = hv % n_low (hv = key * hash_seed, device_hash_function.h:6-18,
device_sketch_v3.h:41-44) belongs to shard floor(b * G / n_low): G contiguous ranges.

Each call is collective: every rank passes its own batch.  insert: each rank partitions its
batch by owner shard (stable, qs_shard_partition), the parts go to their owners in one
all-to-all, and each owner inserts what it received in (source rank, array) order.  That is
the per-bucket order of the ranks' batches concatenated in rank order, so the estimates equal
those of one sketch fed batch 0 of rank 0, batch 0 of rank 1, ..., batch 1 of rank 0, ...
query: the same routing, the owners' estimates return with a second all-to-all and
qs_shard_unpartition puts them back at their array positions.

Every rank holds a sketch of the whole bucket range (its kernels address buckets by their
global number) and touches only its own range; each rank's high pool is its own (n_high
buckets per shard), so a pool that runs out does so per shard.  The exchange runs over
torch.distributed (NCCL between GPUs; gloo in the CPU tests), keys and estimates as int32.
"""
import torch
import torch.distributed as dist

from ._lib import check, lib


def gpu_partition(keys, hash_seed, n_low, n_shards, with_perm, stream=None):
    """Stable partition of a CUDA uint32 batch by owner shard (qs_shard_partition): the
    reordered keys, the per-shard counts (host list) and, with_perm, each output key's index
    in the batch."""
    n = keys.numel()
    out = torch.empty_like(keys)
    perm = torch.empty(n, dtype=torch.int32, device=keys.device) if with_perm else None
    scratch = torch.empty(int(lib.qs_shard_scratch_words(n, n_shards)), dtype=torch.int32, device=keys.device)
    counts = torch.empty(n_shards, dtype=torch.int32, device=keys.device)
    st = (stream or torch.cuda.current_stream()).cuda_stream
    check(lib.qs_shard_partition(keys.data_ptr(), n, hash_seed, n_low, n_shards, out.data_ptr(),
                                 perm.data_ptr() if perm is not None else None, scratch.data_ptr(),
                                 counts.data_ptr(), st), "shard_partition")
    return out, counts.cpu().tolist(), perm


def gpu_unpartition(values, perm, stream=None):
    out = torch.empty_like(values)
    st = (stream or torch.cuda.current_stream()).cuda_stream
    check(lib.qs_shard_unpartition(values.data_ptr(), perm.data_ptr(), values.numel(), out.data_ptr(), st),
          "shard_unpartition")
    return out


class ShardedSketch:
    """MSWS sharded by bucket over `group` (default: the world).  `local` is this rank's
    sketch over the whole bucket range (default: a Sketch_GPU_Sub_Warp_Level built from the
    arguments); `partition(keys, with_perm)` and `unpartition(values, perm)` default to the
    CUDA routing kernels."""

    def __init__(self, n_low, n_high_per_shard, *, hash_seed, mask_table=None, mask_rng=1, group=None, local=None,
                 partition=None, unpartition=None, **knobs):
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        if self.world > 32:
            raise ValueError("at most 32 shards")
        self.n_low, self.hash_seed = int(n_low), int(hash_seed)
        if local is None:
            from .sketch import Sketch_GPU_Sub_Warp_Level
            local = Sketch_GPU_Sub_Warp_Level(n_low, 8, n_high_per_shard, 32, hash_seed=hash_seed,
                                              mask_table=mask_table, mask_rng=mask_rng, **knobs)
        self.local = local
        self._partition = partition or (lambda k, p: gpu_partition(k, self.hash_seed, self.n_low, self.world, p))
        self._unpartition = unpartition or gpu_unpartition

    def owned_buckets(self, shard=None):
        """The bucket range [lo, hi) shard `shard` (default: this rank) owns."""
        g = self.rank if shard is None else shard
        # bucket b belongs to shard floor(b * G / n_low): b from ceil(g * n_low / G) on
        return (g * self.n_low + self.world - 1) // self.world, ((g + 1) * self.n_low + self.world - 1) // self.world

    def _exchange(self, send, counts):
        """All-to-all of a partitioned tensor: returns what this rank received (in source-rank
        order) and the per-source counts."""
        if self.world == 1:
            return send, counts
        dev = send.device
        sc = torch.tensor(counts, dtype=torch.int64, device=dev)
        rc = torch.empty_like(sc)
        dist.all_to_all_single(rc, sc, group=self.group)
        rcounts = rc.cpu().tolist()
        recv = torch.empty(sum(rcounts), dtype=torch.int32, device=dev)
        dist.all_to_all_single(recv, send.view(torch.int32), output_split_sizes=rcounts, input_split_sizes=counts,
                               group=self.group)
        return recv.view(send.dtype), rcounts

    def insert(self, keys):
        """Collective: every rank inserts its batch (uint32 keys on this rank's device)."""
        if self.world == 1:  # one shard owns every bucket: no routing
            self.local.insert(keys)
            return 0
        parts, counts, _ = self._partition(keys, False)
        recv, _ = self._exchange(parts, counts)
        self.local.insert(recv)
        return 0

    def search(self, keys):
        """Collective: estimates of this rank's `keys`, in their order."""
        if self.world == 1:
            return self.local.search(keys)
        parts, counts, perm = self._partition(keys, True)
        recv, rcounts = self._exchange(parts, counts)
        est = self.local.search(recv)
        if self.world > 1:
            back = torch.empty(sum(counts), dtype=torch.int32, device=keys.device)
            dist.all_to_all_single(back, est.view(torch.int32), output_split_sizes=counts,
                                   input_split_sizes=rcounts, group=self.group)
            est = back.view(est.dtype)
        return self._unpartition(est, perm)

    query = search
