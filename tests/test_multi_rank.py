"""Several ranks on the CPU (gloo, world size 2, one process each): the split of the variants
and LM runs over ranks, the gather of the per-variant results in rank order, and a rank that
fails before the gather -- the other rank's collective ends with an error after the process
group's timeout instead of waiting for good. The traced work itself is the oracle's (CPU);
merit_sharded / optimize_lm_sharded, the functions the GPU path runs, are driven with the
oracle's MERIT and the reference's LM in place of the device calls and must give what one rank
gives alone.
"""

import os
import socket
import subprocess
import sys
import textwrap

import numpy as np
import pytest

from mikroptim_b200.multi import partition
from conftest import has_reference_build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = textwrap.dedent("""
    import os, sys, datetime
    sys.path.insert(0, os.environ["MKB_ROOT"])
    import numpy as np
    import torch.distributed as dist
    from mikroptim_b200 import workloads
    from mikroptim_b200.batch import ResidualLayout
    from mikroptim_b200.multi import run_sharded
    import oracle.pyoracle as po

    rank, world, mode = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"]), os.environ["MODE"]
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:" + os.environ["PORT"],
                            rank=rank, world_size=world, timeout=datetime.timedelta(seconds=8))
    b, st, vs, x0 = workloads.singlet(13)
    lay = ResidualLayout(b.topology, st)
    port = po.port()
    if mode == "merit":
        def fn(shard, first):
            m, f, h = port.merit(shard, lay)
            return {"merit": m, "failed": f, "first": np.full(shard.variants, first)}
        out = run_sharded(b, fn)
        m, f, h = port.merit(b, lay)
        assert np.array_equal(out["merit"], m) and np.array_equal(out["failed"], f)
        assert np.array_equal(out["first"][[0, 6, 7, 12]], [0, 0, 7, 7]), out["first"]
    elif mode == "runs":
        one = b.subset(0, 1)
        out = run_sharded(one, lambda shard, first, x: {"x": x * 2.0, "v": np.full(len(x), shard.variants)},
                          x0=x0)
        assert np.array_equal(out["x"], x0 * 2.0) and np.all(out["v"] == 1)
    elif mode == "merit_sharded":
        from mikroptim_b200.multi import merit_sharded
        calls = []

        def oracle_merit(shard, settings):
            calls.append(shard.variants)
            return port.merit(shard, ResidualLayout(shard.topology, settings))
        out = merit_sharded(b, st, merit=oracle_merit)
        m, f, h = port.merit(b, lay)
        assert calls == [7 if rank == 0 else 6], calls
        assert np.array_equal(out["merit"], m) and np.array_equal(out["failed"], f)
        assert np.array_equal(out["hard_failed"], h)
    elif mode == "lm_sharded":
        from mikroptim_b200.multi import optimize_lm_sharded
        ref = po.reference()

        def oracle_lm(shard, layout, vs, x_shard, opt):
            return ref.optimize_lm(shard, layout, vs, x_shard, max_iterations=opt)
        one = b.subset(0, 1)
        out = optimize_lm_sharded(one, lay, vs, x0, options=6, optimize=oracle_lm)
        alone = ref.optimize_lm(one, lay, vs, x0, max_iterations=6)
        for k in ("x", "merit", "status", "iterations", "history"):
            assert np.array_equal(out[k], alone[k]), k
        # uneven runs: every rank gets its own runs' variable sets and padded rows
        ub, ust, uvss, ux0 = workloads.uneven(5, rings=2, spokes=4)
        width = max(v.size for v in uvss)
        seen = []

        def sizes(shard, layout, vs, x_shard, opt):
            seen.append((shard.variants, [v.size for v in vs], x_shard.shape))
            return {"p": np.array([v.size for v in vs]), "x": x_shard + 1.0}
        rows = np.stack([np.pad(np.asarray(r, float), (0, width - len(r))) for r in ux0])
        out = optimize_lm_sharded(ub, ResidualLayout(ub.topology, ust), uvss, rows,
                                  optimize=sizes)
        first = 0 if rank == 0 else 3
        n = 3 if rank == 0 else 2
        assert seen == [(n, [v.size for v in uvss[first:first + n]], (n, width))], seen
        assert np.array_equal(out["p"], [v.size for v in uvss])
        assert np.array_equal(out["x"], rows + 1.0)
    elif mode == "fail":
        if rank == 1:
            raise SystemExit(3)  # leaves before the gather
        try:
            run_sharded(b, lambda shard, first: {"merit": port.merit(shard, lay)[0]})
        except Exception as e:
            print("gather failed:", type(e).__name__)
            raise SystemExit(0)
        raise SystemExit(1)
    dist.destroy_process_group()
    print("ok", rank)
""")


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def launch(mode: str, world: int = 2, timeout: float = 120):
    port = str(free_port())
    procs = []
    for rank in range(world):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE=str(world), PORT=port, MODE=mode,
                   MKB_ROOT=ROOT, MASTER_ADDR="127.0.0.1")
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            out, err = p.communicate(timeout=timeout)
        except subprocess.TimeoutExpired:
            p.kill()
            out, err = p.communicate()
        outs.append((p.returncode, out, err))
    return outs


def test_partition_contiguous_and_balanced():
    for count in (0, 1, 7, 13, 4096):
        for world in (1, 2, 3, 8):
            parts = [partition(count, world, r) for r in range(world)]
            assert sum(n for _, n in parts) == count
            assert all(parts[r][0] + parts[r][1] == parts[r + 1][0] for r in range(world - 1))
            assert max(n for _, n in parts) - min(n for _, n in parts) <= 1
    with pytest.raises(ValueError):
        partition(4, 2, 2)


@pytest.mark.parametrize("mode", ["merit", "runs", "merit_sharded", "lm_sharded"])
def test_two_ranks_gather_in_rank_order(mode):
    if mode == "lm_sharded" and not has_reference_build():
        pytest.skip("reference CPU build not available")
    for rc, out, err in launch(mode):
        assert rc == 0, err[-2000:]
        assert "ok" in out


def test_rank_leaving_before_the_gather_ends_the_other_with_an_error():
    (rc0, out0, err0), (rc1, _, _) = launch("fail")
    assert rc1 == 3
    assert rc0 == 0, err0[-2000:]
    assert "gather failed" in out0
