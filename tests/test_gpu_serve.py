"""Serving form: a request's results are the same whether it is served alone, in a
continuous batch with other requests, or after its network was evicted to the host
and rebuilt.  Deterministic (exact-push) mode, so equality is bit for bit."""
import numpy as np
import pytest

from dtb_b200 import engine as E
from dtb_b200 import network as nw

pytestmark = pytest.mark.gpu

SPECS = [(20_000, 6, 100, 31), (30_000, 8, 200, 32), (15_000, 5, 150, 33), (25_000, 7, 120, 34)]


def _specs():
    return [nw.structured_spec(n, p, k, seed) for n, p, k, seed in SPECS]


def _trace(specs, n_req=10, seed=5, spread=0.004):
    rng = np.random.default_rng(seed)
    reqs, t = [], 0.0
    for _ in range(n_req):
        net = int(rng.integers(len(specs)))
        P = specs[net].n_pops
        ou = (rng.uniform(0.5, 0.7, P).astype(np.float32), rng.uniform(0.15, 0.25, P).astype(np.float32),
              np.full(P, 10.0, np.float32))
        reqs.append(dict(net=net, iters=int(rng.choice([100, 150, 250])), arrival_s=t, ou=ou))
        t += float(rng.uniform(0, spread))
    return reqs


def _solo(specs, reqs):
    """Each network alone through the plain engine path, its requests in arrival order."""
    out = [None] * len(reqs)
    for i, s in enumerate(specs):
        with E.Engine.structured(s, seed=i) as eng:
            for j, r in enumerate(reqs):
                if r["net"] != i:
                    continue
                eng.set_ou(eng.pop_ids, *r["ou"])
                out[j] = eng.run(r["iters"], syn_mode=E.SYN_PUSH_EXACT).freqs
    return out


def _serve(specs, reqs, policy, cap=None, slice_steps=60):
    with E.Server(hbm_cap_bytes=cap, slice_steps=slice_steps, syn_mode=E.SYN_PUSH_EXACT) as srv:
        for i, s in enumerate(specs):
            assert srv.add_structured(s, seed=i) == i
        got = srv.play(reqs, policy)
        return got, srv.info()


def test_batched_requests_equal_solo_runs(gpu):
    specs = _specs()
    reqs = _trace(specs)
    ref = _solo(specs, reqs)
    got, info = _serve(specs, reqs, E.SERVE_BATCHED)
    assert info["batch_members_sum"] > info["slices"]          # requests did share slices
    for j, (g, r) in enumerate(zip(got, ref)):
        assert g["status"] == E.OK
        assert np.array_equal(g["freqs"], r), f"request {j}"
        assert g["finish_s"] >= g["start_s"] >= reqs[j]["arrival_s"]
    assert sum(int(r.sum()) for r in ref) > 0


def test_sequential_policy_equals_batched(gpu):
    specs = _specs()
    reqs = _trace(specs, seed=6)
    a, _ = _serve(specs, reqs, E.SERVE_BATCHED, slice_steps=40)
    b, info = _serve(specs, reqs, E.SERVE_SEQUENTIAL)
    assert info["batch_members_sum"] == info["slices"] == len(reqs)
    for x, y in zip(a, b):
        assert np.array_equal(x["freqs"], y["freqs"])
    # one request at a time: each starts after the previous one finished
    for prev, cur in zip(b, b[1:]):
        assert cur["start_s"] >= prev["finish_s"]


def test_eviction_round_trip_keeps_results(gpu):
    specs = _specs()
    reqs = _trace(specs, n_req=12, seed=7)
    sizes = []
    for i, s in enumerate(specs):
        with E.Engine.structured(s, seed=i) as eng:
            sizes.append(eng.info().device_bytes)
    cap = int(sorted(sizes)[-1] + sorted(sizes)[-2] * 1.05)     # about two networks resident
    ref = _solo(specs, reqs)
    got, info = _serve(specs, reqs, E.SERVE_BATCHED, cap=cap)
    assert info["evictions"] > 0 and info["restores"] > 0
    assert info["resident_bytes"] <= cap
    for g, r in zip(got, ref):
        assert np.array_equal(g["freqs"], r)


@pytest.mark.parametrize("syn,wt", [(E.SYN_PUSH_EXACT, E.W_F32), (E.SYN_PUSH_FIXED, E.W_BF16)], ids=["exact-f32", "fixed-bf16"])
def test_online_requests_from_two_threads_equal_solo_runs(gpu, syn, wt):
    """dtb_server_submit from two client threads while slices run (each thread owns two
    of the networks, so each network's requests keep their order): every request is
    admitted as slots free up and its counts equal the request run alone."""
    import threading
    import time
    specs = _specs()
    reqs = _trace(specs, n_req=16, seed=9)
    solo = [None] * len(reqs)
    for i, s in enumerate(specs):
        with E.Engine.structured(s, seed=i, weight_type=wt) as eng:
            for j, r in enumerate(reqs):
                if r["net"] == i:
                    eng.set_ou(eng.pop_ids, *r["ou"])
                    solo[j] = eng.run(r["iters"], syn_mode=syn).freqs
    got = [None] * len(reqs)
    with E.Server(slice_steps=50, max_batch=3, syn_mode=syn) as srv:
        for i, s in enumerate(specs):
            srv.add_structured(s, seed=i, weight_type=wt)
        srv.start(E.SERVE_BATCHED)

        def client(nets, pause):
            tickets = []
            for j, r in enumerate(reqs):
                if r["net"] in nets:
                    tickets.append((j, srv.submit(r["net"], r["iters"], r["ou"])))
                    time.sleep(pause)
            for j, t in tickets:
                got[j] = srv.wait(t, timeout_s=300)

        threads = [threading.Thread(target=client, args=({0, 1}, 0.004)),
                   threading.Thread(target=client, args=({2, 3}, 0.007))]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        srv.stop()
        info = srv.info()
    assert all(g is not None for g in got)
    assert info["batch_members_sum"] > info["slices"]                  # requests shared slices
    starts = sorted(g["start_s"] for g in got)
    assert any(g["arrival_s"] > starts[0] and g["arrival_s"] < max(x["finish_s"] for x in got) for g in got)
    for j, (g, r) in enumerate(zip(got, solo)):
        assert g["status"] == E.OK
        assert g["finish_s"] >= g["start_s"] >= g["arrival_s"]
        assert np.array_equal(g["freqs"], r), f"request {j}"
    assert sum(int(r.sum()) for r in solo) > 0


def test_online_rejects_and_recovers(gpu):
    specs = _specs()[:1]
    with E.Server(slice_steps=40) as srv:
        srv.add_structured(specs[0], seed=0)
        with pytest.raises(E.DtbError):
            srv.submit(0, 100)                       # not serving yet
        srv.start()
        with pytest.raises(E.DtbError):
            srv.add_structured(specs[0], seed=1)     # networks are added while stopped
        with pytest.raises(E.DtbError):
            srv.play([dict(net=0, iters=10, arrival_s=0.0)])
        t = srv.submit(0, 120)
        r = srv.wait(t)
        assert r["status"] == E.OK and r["freqs"].shape == (120, specs[0].n_pops)
        with pytest.raises(E.DtbError):
            srv.poll(t)                              # already collected
        srv.stop()
        assert srv.add_structured(specs[0], seed=1) == 1
