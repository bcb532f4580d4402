"""Multi-GPU search: reads are independent, so N GPUs each hold a full index and search a contiguous shard
of the input; nothing crosses between GPUs during the search. Shards keep the whole input's bwa batches
and each batch's longest read (batch_max_len), so a shard's reads get exactly the options they would get
in the whole input (src/aln_host.c:23-43), and merging the shards in order gives the single-GPU result.
The reference splits reads over GPUs as read r -> GPU r mod N (src/galn.cu:635); contiguous shards keep
each batch on as few GPUs as possible."""
from __future__ import annotations

import numpy as np

from .api import REC_DTYPE, Reads


def shard_bounds(n: int, world: int) -> list[int]:
    return [n * w // world for w in range(world + 1)]


def batch_ids(reads: Reads) -> np.ndarray:
    n = len(reads)
    return (np.asarray(reads.batch, np.int32) if reads.batch is not None
            else (np.arange(n) // 0x40000).astype(np.int32))


def batch_max_lengths(reads: Reads) -> np.ndarray:
    b = batch_ids(reads)
    lens = np.diff(reads.offset).astype(np.int32)
    out = np.zeros(int(b.max()) + 1 if len(b) else 1, np.int32)
    np.maximum.at(out, b, lens)
    return out


def shard(reads: Reads, rank: int, world: int) -> Reads:
    """This rank's contiguous shard, carrying the whole input's batch ids and longest read per batch."""
    bnd = shard_bounds(len(reads), world)
    lo, hi = bnd[rank], bnd[rank + 1]
    off = reads.offset[lo:hi + 1]
    seq = reads.seq[int(off[0]):int(off[-1])]
    return Reads(seq, (off - off[0]).astype(np.int64), batch_ids(reads)[lo:hi].copy(), batch_max_lengths(reads))


def merge(parts: list[dict]) -> dict:
    """Per-read results of the shards (n_aln, rec_offset, records, pops, trace), in shard order."""
    n_aln = np.concatenate([p["n_aln"] for p in parts]) if parts else np.zeros(0, np.int32)
    recs = np.concatenate([p["records"] for p in parts]) if parts else np.zeros(0, REC_DTYPE)
    off = np.zeros(len(n_aln) + 1, np.int64)
    off[1:] = np.cumsum(np.maximum(n_aln, 0))
    return dict(n_aln=n_aln, rec_offset=off, records=recs,
                pops=np.concatenate([p["pops"] for p in parts]), trace=np.concatenate([p["trace"] for p in parts]))


def sai_bytes(opt_block: bytes, merged: dict) -> bytes:
    out = [b"SAI\x01", bytes(opt_block)]
    for r in range(len(merged["n_aln"])):
        na = max(0, int(merged["n_aln"][r]))
        out.append(np.int32(na).tobytes())
        if na:
            out.append(merged["records"][merged["rec_offset"][r]:merged["rec_offset"][r] + na].tobytes())
    return b"".join(out)


def aln_distributed(search, reads: Reads, rank: int, world: int, group=None) -> dict | None:
    """Run `search(shard) -> dict` on this rank's shard and gather the shards on rank 0 (merged there;
    None on the other ranks). Uses torch.distributed's object gather (gloo or nccl groups)."""
    import torch.distributed as dist
    part = search(shard(reads, rank, world))
    part = {k: np.asarray(part[k]) for k in ("n_aln", "records", "pops", "trace")}
    if world == 1:
        return merge([part])
    got = [None] * world if rank == 0 else None
    dist.gather_object(part, got, dst=0, group=group)
    return merge(got) if rank == 0 else None
