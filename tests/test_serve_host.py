"""Host-side serving logic (no GPU): admission against the byte budget and slot cap."""

from genesis_b200 import serve
from genesis_b200 import workloads as W


def _reqs(n, n_particles=2000, density=32):
    import numpy as np

    rng = np.random.default_rng(0)
    out = []
    for i in range(n):
        sc = W._scene_of(rng, n_particles, density, "elastic", 1e5, 1e-4, 50, f"r{i}")
        out.append(W.Request(i, 0.01 * i, sc))
    return out


def test_admission_is_fifo_within_budget_and_slots():
    reqs = _reqs(5)
    need = serve.estimate_bytes(reqs[0].scene)
    q = serve.AdmissionQueue(budget_bytes=2.5 * need, max_active=10)
    for r in reqs:
        assert q.push(r) is None
    first = q.pop_admissible(0)
    assert [r.rid for r, _ in first] == [0, 1]  # the budget holds two
    assert q.pop_admissible(2) == []
    q.release(first[0][1])
    nxt = q.pop_admissible(1)
    assert [r.rid for r, _ in nxt] == [2]
    q2 = serve.AdmissionQueue(budget_bytes=100 * need, max_active=3)
    for r in reqs:
        q2.push(r)
    assert len(q2.pop_admissible(0)) == 3


def test_oversized_request_is_rejected_up_front():
    reqs = _reqs(1)
    q = serve.AdmissionQueue(budget_bytes=1000, max_active=4)
    assert "more than the whole budget" in q.push(reqs[0])
    assert not q.pending


def test_percentiles_and_sequential_timeline():
    assert serve.percentile([1, 2, 3, 4], 50) == 2.5
    reqs = [W.Request(i, float(i), None) for i in range(3)]
    lat = serve.sequential_timeline(reqs, [2.0, 2.0, 2.0])
    assert lat == [2.0, 3.0, 4.0]
