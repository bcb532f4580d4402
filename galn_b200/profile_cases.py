"""Fixed inputs for profiling one search kernel at a time (ncu captures and timing of a single tier).

    python -m galn_b200.profile_cases warp_steady [--data-dir DIR]

warp_steady: the warp tier in its steady state. From the aDNA workload (100 Mbp reference, 2,000,000 reads,
-l 1024 -n 0.01 -o 2) it takes the first 60,000 reads that the first tier hands to the warp tier and that
need 2,000-50,000 pops: no read long enough to run alone at the end of the launch, so counters describe the
kernel while all warps are busy. They are searched as one bwa batch with -m 100000 (none of them comes near
that cut-off, so their results are those of the full workload) and a 2048-chunk arena per warp (64 Ki
entries), which keeps the device footprint near 4 GB. The search runs twice: the second launch of
warp_kernel is the one to capture (ncu -k regex:warp_kernel -s 1 -c 1). Each run prints its tier times.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np


def warp_steady(data_dir: str) -> None:
    from galn_b200 import Index, Reads, aln, index_build, synth
    os.makedirs(data_dir, exist_ok=True)
    ref, reads, opts = synth.workload("adna", 1.0, seed=1)
    prefix = os.path.join(data_dir, "ref")
    if not os.path.exists(prefix + ".bwt"):
        index_build.build_from_reference(ref, prefix, device="cuda:0")
    full = Reads(reads.ascii(), reads.off.copy())
    ix = Index(prefix)
    ix.set_trace(False)
    sel_path = os.path.join(data_dir, "warp_steady_reads.npy")
    if not os.path.exists(sel_path):
        ix.set_tuning(t0_cap=1024, keep_stats=True)
        r = aln(ix, opts, full)
        prof = ix.last_profile(len(full))
        sel = np.nonzero((prof["tier"] == 1) & (r.pops >= 2000) & (r.pops <= 50000))[0][:60000]
        np.save(sel_path, sel)
    sel = np.load(sel_path)
    sub = Reads.from_strings([bytes(full.seq[full.offset[i]:full.offset[i + 1]]) for i in sel])
    sub.batch = np.zeros(len(sel), np.int32)
    ix.set_tuning(t0_cap=1024, keep_stats=False)
    ix.set_warp_tier(True, 1024)
    args = list(opts) + ["-m", "100000"]
    for _ in range(2):
        r = aln(ix, args, sub)
        p = ix.last_profile()
        print(json.dumps(dict(case="warp_steady", reads=len(sub), ms_tier=[round(x, 3) for x in p["ms_tier"][:2]],
                              pops=int(r.pops.sum()))), flush=True)


CASES = {"warp_steady": warp_steady}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("case", choices=sorted(CASES))
    ap.add_argument("--data-dir", default="/tmp/galn_profile")
    a = ap.parse_args(argv)
    CASES[a.case](a.data_dir)
    return 0


if __name__ == "__main__":
    sys.exit(main())
