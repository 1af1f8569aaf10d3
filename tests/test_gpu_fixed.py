"""The fixed-point push (DTB_SYN_PUSH_FIXED): the float push's kernels with each
step's input summed as packed 32-bit fixed-point fields by integer reductions.

* Against the oracle (models/block_new.py:71-84, W.s summed exactly and rounded
  once): bit for bit whenever every weight is a multiple of the network's unit
  2^-fixed_shift -- U(0,1) float32 weights at in-degree 100 (unit 2^-25), dyadic
  weights at in-degree 1000 (unit 2^-22), in every push variant.
* Deterministic: the same network and noise give the same bits whatever variant
  runs and however the reductions interleave.
* Alone equals mixed: ensemble members advanced in a batch (BF16 weights, graph-
  replayed windows, property updates between windows) and requests served with
  continuous batching give exactly their solo runs' spikes, counts, V and J.
"""
import numpy as np
import pytest

from dtb_b200 import engine as E
from dtb_b200 import network as nw
from oracle import c_oracle as cc
from oracle import lif_oracle as lo

pytestmark = pytest.mark.gpu

VARIANTS = [(E.PUSH_REG, 8), (E.PUSH_REG, 1016), (E.PUSH_TMA, 256), (E.PUSH_LOCAL, 8), (E.PUSH_LOCAL, 2008),
            (E.PUSH_LOCAL, 2016), (E.PUSH_LOCAL, 3008), (-1, 0)]


def _check_against_oracle(eng, net, steps, seed, ou=(0.6, 0.2, 10.0)):
    z, _ = lo.torch_noise_stream(seed, eng.n, steps, False)
    ref = cc.COracle(net, ou=ou)
    sp, counts, ev = ref.run(z)
    eng.set_noise_injected(z)
    r = eng.run(steps, record_spikes=True, syn_mode=E.SYN_PUSH_FIXED)
    assert sp[steps // 2:].mean() > 0.002, "the run must be active"
    assert np.array_equal(r.spikes, sp)
    assert np.array_equal(eng.read_state(E.STATE_V), ref.V)
    assert np.array_equal(eng.read_state(E.STATE_J), ref.J.T)
    assert np.array_equal(eng.read_state(E.STATE_I_OU), ref.i_bg)
    assert r.events == ev


@pytest.mark.parametrize("variant", VARIANTS, ids=[f"{k}:{p}" for k, p in VARIANTS])
def test_block_bit_exact_against_oracle(gpu, variant):
    net = nw.make_uniform_block(10_000, 100, seed=0)
    with E.Engine.from_arrays(net, seed=3) as eng:
        assert eng.info().fixed_shift == 25          # U(0,1) float32 weights are multiples of 2^-24
        eng.set_push_variant(*variant)
        _check_against_oracle(eng, net, 700, seed=1)


@pytest.mark.parametrize("wt", [E.W_F32, E.W_BF16], ids=["f32", "bf16"])
@pytest.mark.parametrize("variant", [(E.PUSH_REG, 8), (E.PUSH_LOCAL, 2008), (E.PUSH_LOCAL, 2016)],
                         ids=["reg:8", "local:2008", "local:2016"])
def test_regional_dyadic_bit_exact_against_oracle(gpu, wt, variant):
    """In-degree 1000 (unit 2^-22): dyadic weights (multiples of 1/256, exact in bf16)."""
    spec = nw.structured_spec(30_000, 10, 1000, seed=5, dyadic_weights=True)
    net = cc.structured_edges(spec)
    with E.Engine.structured(spec, weight_type=wt, seed=2) as eng:
        assert eng.info().fixed_shift == 22 and eng.info().local_windows > 0
        eng.set_push_variant(*variant)
        _check_against_oracle(eng, net, 400, seed=2)


def test_every_variant_gives_the_same_bits(gpu):
    """Philox noise, 1,500 steps of a busy regional network: the order of the integer
    reductions cannot change a bit, so every variant (and the tuner) gives one result."""
    spec = nw.structured_spec(40_000, 12, 500, seed=8)
    results = []
    for variant in [(E.PUSH_REG, 8), (E.PUSH_LOCAL, 2016), (E.PUSH_TMA, 512), (-1, 0)]:
        with E.Engine.structured(spec, weight_type=E.W_BF16, seed=77) as eng:
            eng.set_push_variant(*variant)
            r = eng.run(1500, record_spikes=True, vmean=True, syn_mode=E.SYN_PUSH_FIXED)
            results.append((r.spikes, r.freqs, eng.read_state(E.STATE_V), eng.read_state(E.STATE_J)))
    assert results[0][0][500:].mean() > 0.002
    for other in results[1:]:
        for a, b in zip(results[0], other):
            assert np.array_equal(a, b)


def test_window_graphs_replay_the_same_steps(gpu):
    """Repeated windows of the plain path are captured once and replayed; the result
    equals one long run of the same steps bit for bit."""
    spec = nw.structured_spec(20_000, 8, 300, seed=9)
    with E.Engine.structured(spec, seed=4) as a, E.Engine.structured(spec, seed=4) as b:
        a.set_push_variant(E.PUSH_LOCAL, 2008)
        b.set_push_variant(E.PUSH_LOCAL, 2008)
        fa = [a.run(250, syn_mode=E.SYN_PUSH_FIXED).freqs for _ in range(6)]
        assert a.info().graph_launches >= 4          # windows 3..6 replay the captured graph
        fb = b.run(1500, syn_mode=E.SYN_PUSH_FIXED).freqs
        assert np.array_equal(np.concatenate(fa), fb)
        assert np.array_equal(a.read_state(E.STATE_V), b.read_state(E.STATE_V))
        assert np.array_equal(a.read_state(E.STATE_J), b.read_state(E.STATE_J))


def test_negative_weights_rule_the_mode_out(gpu):
    net = nw.make_uniform_block(2_000, 20, seed=1)
    net["weight"][5, 1] = -0.25
    with E.Engine.from_arrays(net) as eng:
        assert eng.info().fixed_shift == 0
        with pytest.raises(E.DtbError) as ei:
            eng.run(10, syn_mode=E.SYN_PUSH_FIXED)
        assert ei.value.status == E.UNSUPPORTED


MEMBERS = [(20_000, 10, 100, 41), (60_000, 25, 500, 42), (35_000, 14, 200, 43), (90_000, 30, 500, 44)]


def _member_specs():
    rng = np.random.default_rng(4)
    return [nw.structured_spec(n, p, k, s, g_scale=rng.uniform(0.5, 1.5, (p, 4))) for n, p, k, s in MEMBERS]


def test_ensemble_members_equal_their_solo_runs(gpu):
    """The benchmarked ensemble form: BF16 weights, fixed-point push, autotuned,
    graph-replayed 800-step windows with g_AMPA multiplied per population between
    windows (DA_voxel.py:309-353): every member equals its solo run bit for bit."""
    specs = _member_specs()
    windows, W = 4, 800
    g_ampa = E.PROP_IDS["CONDUCT_G_AMPA"]
    rng = np.random.default_rng(7)
    factors = [[rng.uniform(0.97, 1.03, s.n_pops).astype(np.float32) for s in specs] for _ in range(windows)]
    solo = []
    for i, s in enumerate(specs):
        with E.Engine.structured(s, weight_type=E.W_BF16, seed=100 + i) as eng:
            fr = []
            for w in range(windows):
                eng.update_prop_cols([g_ampa] * s.n_pops, np.arange(s.n_pops), factors[w][i])
                fr.append(eng.run(W, syn_mode=E.SYN_PUSH_FIXED).freqs)
            solo.append((np.concatenate(fr), eng.read_state(E.STATE_V), eng.read_state(E.STATE_J)))
    engines = [E.Engine.structured(s, weight_type=E.W_BF16, seed=100 + i) for i, s in enumerate(specs)]
    with E.Batch(engines) as b:
        fr = [[] for _ in specs]
        for w in range(windows):
            for e, s, f in zip(engines, specs, factors[w]):
                e.update_prop_cols([g_ampa] * s.n_pops, np.arange(s.n_pops), f)
            for i, r in enumerate(b.run(W, syn_mode=E.SYN_PUSH_FIXED)):
                fr[i].append(r.freqs)
        assert b.info()["graph_launches"] >= 1
    for i, (f, v, j) in enumerate(solo):
        assert np.array_equal(np.concatenate(fr[i]), f), f"member {i}"
        assert np.array_equal(engines[i].read_state(E.STATE_V), v)
        assert np.array_equal(engines[i].read_state(E.STATE_J), j)
    assert all(f[W:].sum() > 0 for f, _, _ in solo)
    for e in engines:
        e.close()


def test_served_requests_equal_their_solo_runs(gpu):
    """The benchmarked serving form: BF16, fixed-point push, continuous batching
    over slices, requests with new OU parameters: each result equals the request
    run alone on its network."""
    specs = _member_specs()
    rng = np.random.default_rng(11)
    reqs, t = [], 0.0
    for _ in range(12):
        net = int(rng.integers(len(specs)))
        P = specs[net].n_pops
        ou = (rng.uniform(0.55, 0.65, P).astype(np.float32), rng.uniform(0.18, 0.22, P).astype(np.float32),
              np.full(P, 10.0, np.float32))
        reqs.append(dict(net=net, iters=int(rng.choice([300, 500, 800])), arrival_s=t, ou=ou))
        t += float(rng.uniform(0, 0.01))
    solo = [None] * len(reqs)
    for i, s in enumerate(specs):
        with E.Engine.structured(s, weight_type=E.W_BF16, seed=200 + i) as eng:
            for j, r in enumerate(reqs):
                if r["net"] == i:
                    eng.set_ou(eng.pop_ids, *r["ou"])
                    solo[j] = eng.run(r["iters"], syn_mode=E.SYN_PUSH_FIXED).freqs
    with E.Server(slice_steps=100, syn_mode=E.SYN_PUSH_FIXED) as srv:
        for i, s in enumerate(specs):
            srv.add_structured(s, weight_type=E.W_BF16, seed=200 + i)
        got = srv.play(reqs, E.SERVE_BATCHED)
        info = srv.info()
    assert info["batch_members_sum"] > info["slices"]
    for j, (g, r) in enumerate(zip(got, solo)):
        assert g["status"] == E.OK
        assert np.array_equal(g["freqs"], r), f"request {j}"
    assert sum(int(r.sum()) for r in solo) > 0
