"""Host logic of the batch of independent pairs (optflow_b200.batch) on CPU: the seeded batch, the
rank plan, and a world-size-2 gloo run whose gathered results equal a single-process run."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from optflow_b200 import batch


def test_batch_specs_seeded_and_in_range():
    s1, s2 = batch.batch_specs(), batch.batch_specs()
    assert s1 == s2 and len(s1) == 64
    assert {s.w for s in s1} <= set(batch.SIZES) and {s.h for s in s1} <= set(batch.SIZES)
    assert len({(s.w, s.h) for s in s1}) > 10
    for s in s1:
        assert max(abs(s.exx), abs(s.eyy), abs(s.exy)) <= 0.02
        assert np.hypot(s.tx, s.ty) <= 6.0 + 1e-12
        assert 0.003 <= s.noise <= 0.02
    assert batch.batch_specs(seed=12) != s1


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shard_covers_once_and_balances(world):
    specs = batch.batch_specs()
    plan = batch.shard(specs, world)
    flat = sorted(i for p in plan for i in p)
    assert flat == list(range(len(specs)))
    loads = [sum(specs[i].pixels for i in p) for p in plan]
    assert max(loads) - min(loads) <= max(s.pixels for s in specs)
    assert batch.shard(specs, world) == plan


def test_shard_rejects_empty_world():
    with pytest.raises(ValueError):
        batch.shard(batch.batch_specs(4), 0)


def _tiny_pair(spec):
    """A small seeded pair for the CPU run (the GPU renderer is not available here)."""
    rng = np.random.default_rng(spec.seed)
    n = 72 + 8 * (spec.index % 3)
    base = rng.uniform(0, 1, (n + 8, n + 8))
    k = np.exp(-0.5 * (np.arange(-4, 5) / 1.5) ** 2)
    k /= k.sum()
    base = np.apply_along_axis(lambda r: np.convolve(r, k, "same"), 0, base)
    base = np.apply_along_axis(lambda r: np.convolve(r, k, "same"), 1, base)
    a = base[4:4 + n, 4:4 + n].astype(np.float32)
    b = base[3:3 + n, 5:5 + n].astype(np.float32)  # b(x) = a(x + (1, -1)): a moves by (-1, +1) px
    return a, b, None


def _track_oracle(a, b, spec):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(here, "..", "oracle"))
    import oracle
    from optflow_b200 import Config
    r = oracle.track_pair(a, b, Config())
    return np.asarray(r["ux"], np.float32), np.asarray(r["uy"], np.float32)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, specs, out_path):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        local = batch.run_batch(specs, rank, world, _track_oracle, make=_tiny_pair)
        assert set(local) == set(batch.shard(specs, world)[rank])
        merged = batch.gather(local, rank, world)
        if rank == 0:
            np.savez(out_path, **{f"ux{i}": m[0] for i, m in enumerate(merged)},
                     **{f"uy{i}": m[1] for i, m in enumerate(merged)})
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_batch_equals_single_process(tmp_path, oracle):
    specs = batch.batch_specs(6, seed=5)
    out = str(tmp_path / "merged.npz")
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, specs, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = np.load(out)
    single = batch.gather(batch.run_batch(specs, 0, 1, _track_oracle, make=_tiny_pair), 0, 1)
    for i, (ux, uy) in enumerate(single):
        np.testing.assert_array_equal(got[f"ux{i}"], ux)
        np.testing.assert_array_equal(got[f"uy{i}"], uy)
    # the tiny pairs are a (-1, +1) px translation: the tracker found it
    assert abs(np.nanmedian(single[0][0]) + 1.0) < 0.05 and abs(np.nanmedian(single[0][1]) - 1.0) < 0.05
