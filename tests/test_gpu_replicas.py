"""Image write-back (jv_image_set / jv_image_set_device) and the replica
job over a one-rank NCCL group on the GPU."""
import datetime
import socket

import numpy as np
import pytest

from conftest import pkg, rel_l2

pytestmark = pytest.mark.gpu

jv = pkg()


def test_image_set_roundtrip(synth):
    import torch
    s = synth.small_case(n=(14, 12, 10), pml=5, nt=40, seed=2)
    rng = np.random.default_rng(0)
    with jv.Context.from_survey(s) as ctx:
        a = rng.standard_normal((s.nz, s.ny, s.nx))
        ctx.set_image(jv.IMG_PS, a)
        assert np.array_equal(ctx.image(jv.IMG_PS), a)
        d = torch.tensor(rng.standard_normal(a.size), dtype=torch.float64, device="cuda")
        ctx.image_from_device(jv.IMG_SS, d.data_ptr())
        assert np.array_equal(ctx.image(jv.IMG_SS).reshape(-1), d.cpu().numpy())
        e = torch.empty_like(d)
        ctx.image_to_device(jv.IMG_SS, e.data_ptr())
        assert torch.equal(d, e)
        with pytest.raises(jv.JvError):
            ctx.set_image(jv.IMG_PP, a[:-1])
        with pytest.raises(jv.JvError):
            ctx.set_image(7, a)


def test_replica_job_on_one_rank_matches_plain_stack(synth):
    import importlib

    import torch.distributed as dist
    rep = importlib.import_module("domain-decomposition-release_b200.replicas")
    s = synth.small_case(n=(18, 16, 14), pml=5, nt=60, seed=6, shot_idx=[(4, 5, 2), (12, 9, 3), (9, 9, 9)])
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        with jv.Context.from_survey(s) as ctx:
            obs = [ctx.forward(i) for i in range(3)]
            ctx.image_reset()
            for i in range(3):
                ctx.rtm_shot(i, obs[i])
            plain = ctx.images()
            comp0, _ = ctx.finalize()
            mine = rep.run_job(ctx, 3, observed=lambda i: obs[i])
            assert mine == [0, 1, 2]
            rep_img = ctx.images()
            comp1, _ = ctx.finalize()
    finally:
        dist.destroy_process_group()
    for k in plain:
        assert rel_l2(rep_img[k], plain[k]) <= 1e-12
    for k in comp0:
        assert np.array_equal(comp0[k], comp1[k])
