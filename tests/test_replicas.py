"""Multi-rank replica logic on CPU: two gloo ranks on 127.0.0.1.

The GPU path runs the same functions over NCCL (bench.py under torchrun);
here the per-rank work is the oracle codec on each rank's own field, which
is what a replica does on its GPU."""
import os
import socket
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "sc25-stz2_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from stz_b200 import replicas  # noqa: E402


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir, fail_rank):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, os.path.join(ROOT, "sc25-stz2_b200"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    from stz_b200 import fields, replicas as R

    assert R.rank_env() == (rank, rank, world)
    R.init("gloo", timeout_s=20)
    try:
        if rank == fail_rank:
            raise SystemExit(3)  # leaves before the first collective
        # each replica codes the fields it owns; no data crosses ranks
        mine = R.owned(5, rank, world)
        sizes = {}
        for i in mine:
            f = fields.grf((32, 32, 32), 11 / 3, R.replica_seed(100, i), np.float32)
            s = po.compress(f, po.pointwise_eb(f, 1e-3), chunk_high=8, chunk_low=4)
            d = po.decompress(s)
            assert np.abs(d.astype(np.float64) - f).max() <= 1e-3 * (float(f.max()) - float(f.min()))
            sizes[i] = len(s)
        R.barrier()
        t = R.max_over_ranks(10.0 * (rank + 1))
        gbs = R.aggregate_gbs(1e9, R.world_size(), t)
        np.save(os.path.join(out_dir, f"r{rank}.npy"),
                np.array([t, gbs] + [v for _, v in sorted(sizes.items())] + [-1] + mine, np.float64))
    finally:
        R.finalize()


def _spawn(world, tmp_path, fail_rank=-1):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, str(tmp_path), fail_rank)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
        if p.is_alive():
            p.kill()
            p.join()
    return [p.exitcode for p in procs]


def test_owned_partitions_items():
    for world in (1, 2, 3, 8):
        got = sorted(i for r in range(world) for i in replicas.owned(13, r, world))
        assert got == list(range(13))
    with pytest.raises(ValueError):
        replicas.owned(4, 2, 2)


def test_single_process_is_identity():
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.aggregate_gbs(2e9, 1, 1000.0) == pytest.approx(2.0)
    assert replicas.world_size() == 1


def test_two_gloo_ranks(tmp_path):
    codes = _spawn(2, tmp_path)
    assert codes == [0, 0]
    r0 = np.load(tmp_path / "r0.npy")
    r1 = np.load(tmp_path / "r1.npy")
    # max over ranks is the slower rank's time on both ranks
    assert r0[0] == r1[0] == 20.0
    # whole-job throughput: both ranks' bytes over the slowest time
    assert r0[1] == pytest.approx(2 * 1e9 / 0.020 / 1e9)
    # the two replicas owned disjoint fields, covering all five
    own0 = r0[list(r0).index(-1) + 1:].astype(int).tolist()
    own1 = r1[list(r1).index(-1) + 1:].astype(int).tolist()
    assert sorted(own0 + own1) == [0, 1, 2, 3, 4] and not set(own0) & set(own1)


def test_rank_that_leaves_ends_peer_with_error(tmp_path):
    codes = _spawn(2, tmp_path, fail_rank=1)
    assert codes[1] == 3
    # the surviving rank's barrier fails (peer gone / timeout) instead of hanging
    assert codes[0] != 0
    assert not (tmp_path / "r0.npy").exists()
