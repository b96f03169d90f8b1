"""Shot replicas on CPU: world_size-2 gloo process groups drive the host
logic of domain-decomposition-release_b200/replicas.py (shot sharding,
the one image reduction, the write-back before finalize) with a stand-in
context whose "migration" adds a known per-shot pattern.  The CUDA library
is not involved; the stand-in only mimics the Context methods the replica
code calls.  A rank that fails before the reduction ends its peer's
collective with an error instead of a hang."""
import datetime
import socket
import sys
import traceback

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT

sys.path.insert(0, ROOT)


class _Info:
    def __init__(self, n):
        self.n_phy = n


class FakeContext:
    """Host stand-in: shot s migrated adds (s + 1) * (k + 1) * pattern to stack k."""

    def __init__(self, n=1000):
        self.n = n
        self.stacks = np.zeros((5, n))
        self.migrated = []
        self.pattern = np.arange(n, dtype=np.float64) / n

    def info(self):
        return _Info(self.n)

    def image_reset(self):
        self.stacks[:] = 0.0

    def forward(self, s):
        return (np.full(3, s, np.float32),) * 3

    def rtm_shot(self, s, obs):
        assert obs[0][0] == s
        self.migrated.append(s)
        for k in range(5):
            self.stacks[k] += (s + 1) * (k + 1) * self.pattern

    def image(self, k):
        return self.stacks[k].copy()

    def set_image(self, k, arr):
        self.stacks[k] = np.asarray(arr, np.float64).reshape(-1)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, n_shot, fail_rank, q):
    import torch.distributed as dist
    try:
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                                timeout=datetime.timedelta(seconds=20))
        import importlib
        rep = importlib.import_module("domain-decomposition-release_b200.replicas")
        ctx = FakeContext()
        if rank == fail_rank:
            raise RuntimeError("injected failure before the image reduction")
        mine = rep.run_job(ctx, n_shot)
        q.put((rank, "ok", mine, ctx.migrated, ctx.stacks))
        dist.destroy_process_group()
    except Exception as e:  # reported to the parent, which checks it
        q.put((rank, "error", repr(e), traceback.format_exc(), None))


def _run(world, n_shot, fail_rank=-1, timeout=120):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n_shot, fail_rank, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        r = q.get(timeout=timeout)
        out[r[0]] = r
    for p in procs:
        p.join(timeout=30)
        if p.is_alive():
            p.kill()
    return out


def test_shard_shots_covers_every_shot_once():
    import importlib
    rep = importlib.import_module("domain-decomposition-release_b200.replicas")
    for n in (0, 1, 7, 64):
        for w in (1, 2, 3, 8):
            parts = [rep.shard_shots(n, r, w) for r in range(w)]
            flat = sorted(s for p in parts for s in p)
            assert flat == list(range(n))
            assert max(map(len, parts)) - min(map(len, parts)) <= 1
    with pytest.raises(ValueError):
        rep.shard_shots(4, 2, 2)


@pytest.mark.parametrize("n_shot", [5, 2, 1])
def test_two_rank_job_sums_images_of_all_shots(n_shot):
    out = _run(2, n_shot)
    pattern = np.arange(1000, dtype=np.float64) / 1000
    want = np.stack([sum((s + 1) for s in range(n_shot)) * (k + 1) * pattern for k in range(5)])
    seen = []
    for r in (0, 1):
        rank, status, mine, migrated, stacks = out[r]
        assert status == "ok", migrated
        assert mine == migrated == list(range(r, n_shot, 2))
        seen += migrated
        np.testing.assert_allclose(stacks, want, rtol=0, atol=1e-12)
    assert sorted(seen) == list(range(n_shot))


def test_failed_rank_ends_peer_collective_with_error():
    out = _run(2, 4, fail_rank=1, timeout=90)
    assert out[1][1] == "error" and "injected failure" in out[1][2]
    assert out[0][1] == "error"  # the peer's all_reduce ended with an error, not a hang
