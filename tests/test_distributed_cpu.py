"""The multi-rank path on CPU: two gloo ranks (world size 2) take the reference's
job split of the search positions, gather their worker result arrays on rank 0
and merge them there as the master does; the merge equals the single-process
merge of the same arrays, and the timing helpers bench.py uses (barrier, max
over ranks) agree across ranks."""
import math
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _maps(seed, nx, ny):
    rng = np.random.default_rng(seed)
    m = {k: rng.normal(size=(ny, nx)).astype(np.float32) for k in
         ("mip", "psi", "theta", "phi", "defocus", "pixel", "sum", "sumsq")}
    m["mip"] = np.abs(m["mip"]) + np.float32(0.1)
    m["sumsq"] = np.abs(m["sumsq"]) * np.float32(10) + np.float32(5)
    return m, rng.integers(0, 1000, size=512)


def _worker(rank, world, port, out_dir, mismatch):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist
    from cistem_downstream_bah_b200 import distributed as D
    from cistem_downstream_bah_b200 import hostprep as H
    w, r, _ = D.init_from_env("gloo", timeout_s=60)
    assert (w, r) == (world, rank)
    try:
        D.barrier(w)
        mx = D.max_over_ranks(w, float(rank + 1) * 1.5)
        sm = D.sum_over_ranks(w, float(rank + 1))
        first, last = D.rank_search_range(1595, r, w)
        nx = 36 if not (mismatch and rank == 1) else 34
        maps, hist = _maps(100 + rank, nx, 30)
        arr = H.pack_worker_result(maps, nx, 30, 0, float(last - first + 1) * 241, math.sqrt(nx * 30), hist)
        np.save(os.path.join(out_dir, f"arr{rank}.npy"), arr)
        try:
            merged = D.gather_merge(arr)
            status = "ok"
        except ValueError:
            merged, status = None, "mismatch"
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(f"{mx} {sm} {first} {last} {status}\n")
        if merged is not None:
            np.savez(os.path.join(out_dir, "merged.npz"), **{k: v for k, v in merged.items() if isinstance(v, np.ndarray)},
                     expected_threshold=merged["expected_threshold"], number_of_ccs=merged["number_of_ccs"])
    finally:
        dist.destroy_process_group()


def _spawn(tmp_path, mismatch=False):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, str(tmp_path), mismatch)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    for p in procs:
        if p.is_alive():
            p.kill()
            p.join()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    return [open(tmp_path / f"rank{r}.txt").read().split() for r in range(2)]


def test_two_gloo_ranks_gather_and_merge_like_the_master(tmp_path):
    from cistem_downstream_bah_b200 import hostprep as H
    lines = _spawn(tmp_path)
    ranges = H.job_search_ranges(1595, 2)
    for r, ln in enumerate(lines):
        assert float(ln[0]) == 3.0 and float(ln[1]) == 3.0
        assert (int(ln[2]), int(ln[3])) == ranges[r]
        assert ln[4] == "ok"
    arrays = [np.load(tmp_path / f"arr{r}.npy") for r in range(2)]
    ref = H.merge_results(arrays)
    got = np.load(tmp_path / "merged.npz")
    for k in H.MASTER_MAPS + ("rows",):
        assert np.array_equal(got[k], ref[k]), k
    assert float(got["number_of_ccs"]) == ref["number_of_ccs"] == 1595 * 241
    assert float(got["expected_threshold"]) == ref["expected_threshold"]


def test_mismatching_arrays_fail_on_every_rank(tmp_path):
    lines = _spawn(tmp_path, mismatch=True)
    assert [ln[4] for ln in lines] == ["mismatch", "mismatch"]
    assert not (tmp_path / "merged.npz").exists()
