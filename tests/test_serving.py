"""Serving loop (uc_server_*): each job's lines are the same alone and in a
mix of concurrently admitted, batched and overlapping jobs; admission keeps
the pool within its budget; a job larger than the pool fails cleanly."""
import threading

import pytest
import torch

from tests.cases import sorted_lines

pytestmark = pytest.mark.gpu


def _jobs(count, scale):
    from unitigcoarsening_b200 import synth
    out = []
    for j in range(count):
        spec, k = synth.served_job(j, seed=9, scale=scale)
        out.append((synth.make_text(spec, k).numpy().tobytes(), k))
    return out


@pytest.fixture(scope="module")
def mix():
    return _jobs(24, 0.004)  # 40 to 200k k-mers each, k = 31 or 63


def test_results_same_alone_and_in_mix(comp, mix):
    from unitigcoarsening_b200 import Server
    alone = [sorted_lines(bytes(comp.compact_host(t, k, min(8, k - 1)).numpy())) for t, k in mix]
    with Server(lanes=3, max_batch=8, hbm_budget=3 << 30) as srv:
        tickets = [srv.submit(t, k, min(8, k - 1)) for t, k in mix]  # a burst: jobs queue behind busy lanes
        res = [srv.wait(t, timeout=120) for t in tickets]
        st = srv.stats()
    for (data, info), want, (t, k) in zip(res, alone, mix):
        assert info["status"] == 0
        assert sorted_lines(data) == want
        assert info["latency_ms"] >= info["queue_ms"] >= 0
        assert info["n_kmers"] == int(t[: t.index(b"\n")])
    assert st["jobs_done"] == len(mix)
    assert st["kmers_done"] == sum(int(t[: t.index(b"\n")]) for t, _ in mix)
    assert st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
    assert st["batches"] >= 1 and st["batched_jobs"] >= 2  # queued small jobs were merged
    assert st["pool_peak_bytes"] <= st["pool_bytes"]


def test_matches_oracle_under_concurrent_submitters(comp, oracle, mix):
    from unitigcoarsening_b200 import Server
    sub = mix[:8]
    want = [sorted_lines(oracle.compact(t, k)[0]) for t, k in sub]
    got = [None] * len(sub)
    with Server(lanes=2, max_batch=4, hbm_budget=2 << 30) as srv:
        def client(i):
            t, k = sub[i]
            got[i] = srv.wait(srv.submit(t, k, min(8, k - 1)), timeout=120)[0]
        th = [threading.Thread(target=client, args=(i,)) for i in range(len(sub))]
        for x in th:
            x.start()
        for x in th:
            x.join()
    for g, w in zip(got, want):
        assert sorted_lines(g) == w


def test_admission_under_a_small_pool(comp, mix):
    """A pool that holds only a few jobs at once: jobs wait for memory,
    none fails, the peak stays within the pool."""
    from unitigcoarsening_b200 import Server, UCError
    sub = [(t, k) for t, k in mix if k == 31][:10]
    alone = [sorted_lines(bytes(comp.compact_host(t, k, 8).numpy())) for t, k in sub]
    budget = 160 << 20
    with Server(lanes=4, max_batch=1, hbm_budget=budget) as srv:
        tickets = [srv.submit(t, k, 8) for t, k in sub]
        res = [srv.wait(t, timeout=120) for t in tickets]
        st = srv.stats()
        from unitigcoarsening_b200 import synth
        huge = synth.make_text(synth.GenomeSpec(length=3_000_000, gc=0.5, seed=3), 31).numpy().tobytes()
        t_big = srv.submit(huge, 31, 8)
        with pytest.raises(UCError) as ei:
            srv.wait(t_big, timeout=120)
        assert ei.value.status == 3  # UC_EBUDGET: its footprint exceeds the pool
    for (data, _), want in zip(res, alone):
        assert sorted_lines(data) == want
    assert st["pool_peak_bytes"] <= budget


def test_bad_job_fails_alone(comp, mix):
    """A job whose count line disagrees with its lines, and one with a line
    shorter than k, fail with UC_EINPUT; the jobs around them (batched or
    not) complete with their own lines."""
    from unitigcoarsening_b200 import Server, UCError
    good = [(t, k) for t, k in mix if k == 31][:6]
    alone = [sorted_lines(bytes(comp.compact_host(t, k, 8).numpy())) for t, k in good]
    t0 = good[0][0]
    head, body = t0.split(b"\n", 1)
    wrong_count = str(int(head) + 5).encode() + b"\n" + body
    short_line = b"2\n" + b"A" * 31 + b"\nACGT\n"
    jobs = [good[0], (wrong_count, 31), good[1], good[2], (short_line, 31), good[3], good[4], good[5]]
    with Server(lanes=2, max_batch=4, hbm_budget=2 << 30) as srv:
        tickets = [srv.submit(t, k, 8) for t, k in jobs]
        results = []
        for t in tickets:
            try:
                results.append(srv.wait(t, timeout=120)[0])
            except UCError as e:
                results.append(e.status)
    assert results[1] == 1 and results[4] == 1  # UC_EINPUT
    got = [r for i, r in enumerate(results) if i not in (1, 4)]
    for g, w in zip(got, alone):
        assert sorted_lines(g) == w
