"""Multi-rank host logic on CPU: world_size-2 `gloo` process group (no GPU).

Checks the k sharding (every k exactly once, contiguous, balanced), max-over-ranks step time, global
sums, and the kept-list offsets of the window filter: two ranks that each filter their own k shard and
place their kept indices at the all-gathered offsets reproduce the single-process kept list exactly.
"""
import os
import socket

import numpy as np
import pytest

from epb200 import shard


def test_shard_range_partition():
    for n in (0, 1, 7, 2048, 2049):
        for w in (1, 2, 3, 8):
            ranges = [shard.shard_range(n, w, r) for r in range(w)]
            assert ranges[0][0] == 0 and ranges[-1][1] == n
            for (a, b), (c, d) in zip(ranges[:-1], ranges[1:]):
                assert b == c
            sizes = [b - a for a, b in ranges]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard.shard_range(10, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_dir):
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    for p in (os.path.dirname(here), os.path.join(os.path.dirname(here), "electronphonon.jl_b200")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import datetime

    import torch.distributed as dist

    from epb200 import shard as S
    from oracle import epb_oracle as O

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        rng = np.random.default_rng(0)
        nk, nw = 1001, 6
        E = np.sort(rng.normal(size=(nw, nk)), axis=0)  # the same "band energies" on every rank
        a, b = S.shard_range(nk, world, rank)
        local = [k for k in range(a, b) if O.inside_window(E[:, k], -0.1, 0.05)[1] >= O.inside_window(E[:, k], -0.1, 0.05)[0]]
        off, total = S.global_offsets(len(local))
        glob = np.full(total, -1, dtype=np.int64)
        glob[off:off + len(local)] = local
        t = S.max_over_ranks(1.5 + rank)
        s = S.sum_over_ranks(float(len(local)))
        np.save(os.path.join(out_dir, f"r{rank}.npy"), np.array([off, total, t, s] + list(glob)))
    finally:
        dist.destroy_process_group()


def test_gloo_world2_window_offsets(tmp_path):
    import torch.multiprocessing as mp

    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    from oracle import epb_oracle as O

    rng = np.random.default_rng(0)
    E = np.sort(rng.normal(size=(6, 1001)), axis=0)
    ref = [k for k in range(1001) if O.inside_window(E[:, k], -0.1, 0.05)[1] >= O.inside_window(E[:, k], -0.1, 0.05)[0]]
    r0, r1 = (np.load(tmp_path / f"r{r}.npy") for r in range(2))
    total = int(r0[1])
    assert total == int(r1[1]) == len(ref)
    assert r0[2] == r1[2] == 2.5          # max over ranks
    assert r0[3] == r1[3] == len(ref)     # global sum
    g = np.where(r0[4:] >= 0, r0[4:], r1[4:]).astype(np.int64)
    np.testing.assert_array_equal(g, ref)


def _sigma_worker(rank, world, port, out_dir):
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    for p in (os.path.dirname(here), os.path.join(os.path.dirname(here), "electronphonon.jl_b200")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import datetime

    import torch.distributed as dist

    from epb200 import bte

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sig = np.arange(9, dtype=np.float64).reshape(3, 3, order="F") * (rank + 1)
        st = dict(kept_k=10, states=3 + rank, pairs=100 * (rank + 1), width=2)
        tot, st2 = bte.reduce_shards(sig, st)
        np.save(os.path.join(out_dir, f"s{rank}.npy"),
                np.array(list(tot.reshape(-1, order="F")) + [st2["pairs"], st2["states"], st2["kept_k"], st2["width"]]))
    finally:
        dist.destroy_process_group()


def test_gloo_world2_bte_shard_reduction(tmp_path):
    """The SERTA consumer's k shards: sigma (partial sums) and the pair / state counts add over the ranks;
    the kept-k count and the window width are common."""
    import torch.multiprocessing as mp

    port = _free_port()
    mp.start_processes(_sigma_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    r0, r1 = (np.load(tmp_path / f"s{r}.npy") for r in range(2))
    np.testing.assert_array_equal(r0, r1)
    np.testing.assert_array_equal(r0[:9], np.arange(9) * 3.0)
    assert list(r0[9:]) == [300, 7, 10, 2]
