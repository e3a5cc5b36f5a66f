"""Multi-process rank plumbing (openvort_b200.dist, openvort_b200.shard) on
CPU with gloo, world size 2: the timing collectives of multi-GPU runs, the
per-rank seeds of the independent tangles, the in-place exchange of a
tangle sharded over ranks, and a rank that never joins a collective ending
the other's with an error (host-side failure detection)."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
mp = pytest.importorskip("torch.multiprocessing")


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q, mode):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    from openvort_b200 import dist as D
    try:
        r = D.setup("gloo", timeout_s=5.0)
        if mode == "collectives":
            D.barrier(r)
            mx = D.max_over_ranks(r, 1.5 + rank)
            sm = D.sum_over_ranks(r, 1.0 + rank)
            q.put((rank, mx, sm, D.rank_seed(2024, rank), D.describe(r)))
        elif mode == "exchange":
            # sharded evaluations: each rank's block of the exchange buffer,
            # all-gathered in place; the tail beyond world * block untouched
            from openvort_b200.shard import exchange
            block = 7
            xbuf = torch.full((world * block + 3,), -1.0, dtype=torch.float64)
            xbuf[rank * block:(rank + 1) * block] = torch.arange(block, dtype=torch.float64) + 100 * rank
            exchange(xbuf, r, block)
            q.put((rank, xbuf.tolist()))
        elif mode == "sharded_run":
            # ShardedRun's loop with a stand-in for the device state: at
            # begin each rank writes its block, at end every block must be
            # there; 4 stages per step, buffer sized by shard_bytes
            from openvort_b200.shard import ShardedRun

            class Stand:
                n_active = 11
                seen = []

                def shard_bytes(self, world):
                    return 48 * (-(-self.n_active // world)) * world

                def shard(self, rank_, world_, ptr, nbytes):
                    self.nbytes = nbytes

                def shard_begin(self, q, t, dt):
                    b = run.block
                    run.xbuf[rank * b:(rank + 1) * b] = 1000 * q + 10 * rank + torch.arange(b)

                def shard_end(self, q, t, dt):
                    b = run.block
                    want = torch.cat([1000 * q + 10 * rr + torch.arange(b) for rr in range(world)])
                    self.seen.append((q, bool(torch.equal(run.xbuf[:world * b], want.double()))))

            stand = Stand()
            run = ShardedRun(stand, r)
            run.run(0.0, 1e-6, 2)
            q.put((rank, stand.nbytes, run.block, stand.seen))
        elif mode == "missing_rank":
            if rank == 1:
                q.put((rank, "left"))           # leaves between steps, joins nothing
            else:
                try:
                    D.max_over_ranks(r, 1.0)
                    q.put((rank, "no error"))
                except Exception as e:          # the group's timeout ends the collective
                    q.put((rank, "error", type(e).__name__))
        if mode != "missing_rank":
            D.close(r)
    except Exception as e:   # pragma: no cover - reported to the parent
        q.put((rank, "exception", repr(e)))


def _run(mode, world=2, timeout=60):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, mode)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=timeout) for _ in range(world)]
    for p in procs:
        p.join(timeout=timeout)
        if p.is_alive():
            p.kill()
    return sorted(out)


def test_single_process_needs_no_group(monkeypatch):
    from openvort_b200 import dist as D
    monkeypatch.delenv("WORLD_SIZE", raising=False)
    r = D.setup()
    assert r.world == 1 and r.pg is None
    assert D.max_over_ranks(r, 3.0) == 3.0
    assert D.describe(r) == {"backend": None, "world": 1}
    D.barrier(r)


def test_timing_collectives_world_2():
    out = _run("collectives")
    assert [o[0] for o in out] == [0, 1]
    for rank, mx, sm, seed, pg in out:
        assert mx == 2.5          # the slowest rank's time
        assert sm == 3.0
        assert seed == 2024 + 1000 * rank
        assert pg == {"backend": "gloo", "world": 2}
    assert out[0][3] != out[1][3]  # every rank its own tangle


def test_rank_that_never_joins_ends_the_collective_with_an_error():
    out = _run("missing_rank")
    assert out[1][:2] == (1, "left")
    assert out[0][0] == 0 and out[0][1] == "error"


def test_shard_exchange_world_2():
    """The in-place all-gather between ov_state_shard_begin and _end: after
    it every rank holds every rank's block, in rank order."""
    out = _run("exchange")
    block = 7
    want = [float(i + 100 * r) for r in range(2) for i in range(block)] + [-1.0] * 3
    assert [o[0] for o in out] == [0, 1]
    for _, got in out:
        assert got == want


def test_sharded_run_loop_world_2():
    """ShardedRun.step: begin, the exchange, then end for each of the 4
    stages; at every end all ranks' blocks are in the buffer."""
    out = _run("sharded_run")
    for rank, nbytes, block, seen in out:
        assert nbytes == 48 * 6 * 2 and block == 6 * 6
        assert seen == [(q, True) for _ in range(2) for q in range(4)]
