"""Shot sharding and the cross-rank stack, as world_size-2 gloo ranks on CPU.

The device halves (``ertm_stack_partial`` / ``ertm_stack_finish``) are replaced
by NumPy stand-ins here, so these tests cover the plan, the status exchange and
the all-reduce of the float64 partial stacks; the GPU parity tests cover the
device halves."""

from __future__ import annotations

import datetime
import socket
import types

import numpy as np
import pytest

import oracle
from ertm_b200.parallel import ShardError, ShardResult, ShotParallelMigrator, exchange_status, plan_shards, \
    reduce_partial_sums, shot_cost

NZ, NX = 23, 31


def _images(n_shots: int, n_modes: int) -> list[list[np.ndarray]]:
    rng = np.random.default_rng(11)
    return [[(rng.standard_normal((NZ, NX)) * (1 + 3 * i + k)).astype(np.float32) for k in range(n_modes)]
            for i in range(n_shots)]


def _job(n_shots: int, nt=lambda i: 100 + 10 * i):
    grid = types.SimpleNamespace(nx=NX, nz=NZ, shape=(NZ, NX))
    model = types.SimpleNamespace(grid=grid)
    shots = [types.SimpleNamespace(index=i, data=np.zeros((nt(i), 4), np.float32)) for i in range(n_shots)]
    imager = types.SimpleNamespace(config=types.SimpleNamespace(mode="pp"),
                                   solver_config=types.SimpleNamespace(engine="elastic"))
    return imager, shots, model


def _fake_local(images, fail_rank=None, rank=None):
    import torch

    def local(shots, models, modes, wavelets, normalize):
        if fail_rank is not None and rank == fail_rank:
            raise RuntimeError("planted failure in this rank's shard")
        partial = np.zeros((len(modes), NZ, NX), dtype=np.float64)
        per_shot = []
        for s in shots:
            res = []
            for k in range(len(modes)):
                d = images[s.index][k].astype(np.float64)
                if normalize:
                    m = float(np.max(np.abs(d)))
                    if m > 0:
                        d = d / m
                partial[k] += d
                res.append(types.SimpleNamespace(meta={"engine": "elastic"}))
            per_shot.append(res)
        return ShardResult(torch.from_numpy(partial), len(shots), per_shot)
    return local


def _fake_finish(total, count):
    return (total.numpy() / count).astype(np.float32)


# ---------------------------------------------------------------------------
# the plan (no processes)
# ---------------------------------------------------------------------------
def test_plan_equal_costs_round_robin():
    assert plan_shards([1.0] * 8, 2) == [[0, 2, 4, 6], [1, 3, 5, 7]]
    assert plan_shards([1.0] * 3, 4) == [[0], [1], [2], []]
    assert plan_shards([5.0], 1) == [[0]]


def test_plan_largest_first_balances_load():
    costs = [shot_cost(nx, nz, nt, "elastic") for nx, nz, nt in
             [(501, 301, 1500), (2401, 1201, 6000), (1001, 501, 3000), (1601, 801, 2000), (501, 301, 6000),
              (2401, 1201, 1500)]]
    plan = plan_shards(costs, 3)
    assert sorted(i for s in plan for i in s) == list(range(len(costs)))
    loads = [sum(costs[i] for i in s) for s in plan]
    # greedy largest-first is within 4/3 of the optimum, itself >= max(cost, mean load)
    bound = max(max(costs), sum(costs) / 3)
    assert max(loads) <= 4.0 / 3.0 * bound + 1e-6
    assert plan == plan_shards(list(costs), 3)        # deterministic


def test_plan_rejects_empty_world():
    with pytest.raises(ValueError):
        plan_shards([1.0], 0)


def test_single_process_job_matches_oracle_stack():
    imager, shots, model = _job(5)
    imgs = _images(5, 2)
    m = ShotParallelMigrator(imager, local=_fake_local(imgs), finish=_fake_finish)
    out = m.migrate_job(shots, model, modes=("pp", "ps"))
    for k in range(2):
        ref = oracle.stack_images([imgs[i][k] for i in range(5)], normalize=True)
        assert np.array_equal(out[k].image, ref)
        assert out[k].meta["n_shots"] == 5 and out[k].meta["ranks"] == 1


def test_single_shot_job_is_the_image_itself():
    imager, shots, model = _job(1)
    imgs = _images(1, 1)
    out = ShotParallelMigrator(imager, local=_fake_local(imgs), finish=_fake_finish).migrate_job(shots, model)
    assert np.array_equal(out[0].image, imgs[0][0])
    assert out[0].meta["stack_normalize"] is False


# ---------------------------------------------------------------------------
# two gloo ranks
# ---------------------------------------------------------------------------
def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, scenario: str, n_shots: int, q) -> None:
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        imager, shots, model = _job(n_shots)
        imgs = _images(n_shots, 2)
        if scenario == "status":
            q.put((rank, exchange_status(rank == 1), exchange_status(False)))
        elif scenario == "sum":
            import torch
            t = torch.full((3, 4), float(rank + 1), dtype=torch.float64)
            q.put((rank, reduce_partial_sums(t).numpy().tolist()))
        elif scenario == "job":
            m = ShotParallelMigrator(imager, local=_fake_local(imgs), finish=_fake_finish)
            out = m.migrate_job(shots, model, modes=("pp", "ps"))
            q.put((rank, [o.image for o in out], out[0].meta["shard"]))
        elif scenario == "fail":
            m = ShotParallelMigrator(imager, local=_fake_local(imgs, fail_rank=1, rank=rank), finish=_fake_finish)
            try:
                m.migrate_job(shots, model, modes=("pp",))
                q.put((rank, "no error"))
            except ShardError as exc:
                q.put((rank, str(exc)))
    finally:
        dist.destroy_process_group()


def _run(scenario: str, n_shots: int = 7, world: int = 2):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, scenario, n_shots, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        item = q.get(timeout=120)
        out[item[0]] = item[1:]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return out


def test_gloo_status_exchange():
    out = _run("status")
    assert out[0] == (1, 0) and out[1] == (1, 0)


def test_gloo_partial_sum_all_reduce():
    out = _run("sum")
    assert out[0][0] == out[1][0] == [[3.0] * 4] * 3


def test_gloo_sharded_job_equals_one_process_stack():
    n = 7
    out = _run("job", n_shots=n)
    imgs = _images(n, 2)
    shards = [out[r][1] for r in range(2)]
    assert sorted(shards[0] + shards[1]) == list(range(n)) and not set(shards[0]) & set(shards[1])
    for k in range(2):
        ref = oracle.stack_images([imgs[i][k] for i in range(n)], normalize=True)
        for r in range(2):
            np.testing.assert_allclose(out[r][0][k], ref, rtol=1e-6, atol=1e-7)
        assert np.array_equal(out[0][0][k], out[1][0][k])


def test_gloo_failed_shard_raises_on_every_rank():
    out = _run("fail")
    for r in range(2):
        assert "1 of 2 rank(s) failed" in out[r][0]


def test_gloo_more_ranks_than_shots():
    out = _run("job", n_shots=1)
    imgs = _images(1, 2)
    for r in range(2):
        assert np.array_equal(out[r][0][0], imgs[0][0])
