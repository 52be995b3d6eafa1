"""The host table workers of streamed corrector training: every job comes back once, also when a
worker process dies mid-stream (killed here on purpose; CPU only)."""
import os
import signal

from fvm_solver_b200 import batched as B


def test_table_workers_survive_a_dead_worker():
    pool = B.TableWorkers(2)
    try:
        jobs = {i: (i, 1234, "channel", (300_000, 800_000)) for i in range(6)}
        for i, job in jobs.items():
            pool.submit(i, job)
        first = pool.get(0)
        os.kill(pool.procs[0].pid, signal.SIGKILL)       # a worker dies with jobs still queued
        got = {0: first, **{i: pool.get(i, timeout=300) for i in range(1, 6)}}
        assert pool.restarts >= 1 and -signal.SIGKILL in pool.exit_codes
        for i in jobs:
            want = B._ensemble_worker(jobs[i])
            assert got[i].kt.n_cells == want.kt.n_cells and got[i].name == want.name
        assert not pool.pending
    finally:
        pool.close()
