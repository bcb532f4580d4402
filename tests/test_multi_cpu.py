"""The multi-GPU host path on CPU: two gloo ranks each search their contiguous shard (with the oracle
standing in for a GPU), and the merged result equals the whole input's, byte for byte, against the
reference's golden .sai -- including a case whose bwa batches straddle the shard boundary."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle
from conftest import GOLDEN, case_paths, golden_cases


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, name, out_dir):
    import torch.distributed as dist

    import galn_b200
    from galn_b200 import multi
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    meta = golden_cases()[name]
    p = case_paths(name, meta)
    reads = galn_b200.read_fastq(p["fq"])
    ob = oracle.opt_bytes(oracle.parse_aln_args(meta["opts"]))
    idx = oracle.Index(os.path.join(GOLDEN, meta["ref"], "ref.bwt"))

    def search(sh):
        q = oracle.encode_queries(sh.seq, sh.offset)
        r = oracle.aln(idx, ob, q, sh.offset, np.diff(sh.offset).astype(np.int32), sh.batch, 1,
                       batch_max_len=sh.batch_max_len)
        return dict(n_aln=r.n_aln, records=r.records, pops=r.pops, trace=r.trace)

    merged = multi.aln_distributed(search, reads, rank, world)
    if rank == 0:
        with open(os.path.join(out_dir, name + ".sai"), "wb") as f:
            f.write(multi.sai_bytes(ob, merged))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("name", ["adna", "edge_default", "edge_loggap"])
def test_two_rank_shards_merge_to_the_reference(name, tmp_path):
    oracle.build()
    mp.spawn(_rank, args=(2, _free_port(), name, str(tmp_path)), nprocs=2, join=True)
    got = open(tmp_path / (name + ".sai"), "rb").read()
    assert got == open(case_paths(name, golden_cases()[name])["sai"], "rb").read()


def test_shard_carries_whole_input_batches():
    import galn_b200
    from galn_b200 import multi
    seqs = ["A" * 10] * 5 + ["C" * 90] + ["G" * 20] * 4
    reads = galn_b200.Reads.from_strings(seqs)
    reads.batch = np.array([0] * 6 + [1] * 4, np.int32)
    s0, s1 = multi.shard(reads, 0, 2), multi.shard(reads, 1, 2)
    assert list(s0.batch_max_len) == [90, 20] and list(s1.batch_max_len) == [90, 20]
    assert len(s0) + len(s1) == 10 and list(s1.batch) == [0, 1, 1, 1, 1]
