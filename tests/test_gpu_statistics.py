"""The benchmarked production path against the oracle at the statistical bar:
population firing rates within 2 % and pooled ISI CV within 5 % over 10,000
steps (models/block_new.py:122-158, the OU draw :92-96).

The production path is the float push (red.global vector reductions and the
population-local shared-memory windows, autotuned or forced to the variants the
5M-neuron bench picks), FP32 and BF16 weights, with Philox OU noise.  Three
networks:

* ``block10k``   -- the plain 10k block, in-degree 100 (168.7 Hz in the oracle);
* ``quiet50k``   -- a 50k-neuron regional network, 10 populations, in-degree 1000,
                    receptor conductances x 0.01 and OU mean 0.65: 7.9 Hz, far below
                    the refractory ceiling;
* ``busy50k``    -- the same construction at the bench's parameters: every
                    population at the refractory ceiling, 197.8 Hz.

Two comparisons:

* paired -- the engine consumes the oracle's own noise stream (torch seed 0,
  injected), so the two runs differ only in how the synaptic input is summed
  (float reductions in any order, window fixed point, BF16 weights).  Both bars
  are asserted as stated: every population's rate within 2 %, pooled ISI CV
  within 5 % (FP32 vs BF16 oracles on the same stream agree to 0.25 % / 0.8 %).
* unpaired -- the engine draws its own Philox noise.  Two independent noise
  realizations of the reference model itself disagree by more than the bar on
  some statistics (block10k's ISI CV spreads 2.3 % (1 sigma) over ten torch
  seeds, quiet50k's single-population rates about 2 %), so each statistic is held
  to the bar or to four times the oracle's own seed-to-seed spread, whichever is
  wider, around the mean of several oracle seeds.

Every test prints one ``STATS {json}`` line with the measured margins.
"""
import json

import numpy as np
import pytest

from dtb_b200 import engine as E
from dtb_b200 import network as nw
from oracle import c_oracle as cc
from oracle import lif_oracle as lo
from tests.spike_stats import IsiMoments, population_rates

pytestmark = pytest.mark.gpu

STEPS, WARM, CHUNK, DT = 10_000, 1_000, 1_000, 0.1
RATE_BAR, CV_BAR = 0.02, 0.05

NETWORKS = {
    "block10k": dict(kind="uniform", n=10_000, k=100, ou=(0.6, 0.2, 10.0), seeds=10),
    "quiet50k": dict(kind="regional", n=50_000, P=10, k=1000, g=0.01, ou=(0.65, 0.2, 10.0), seeds=3),
    "busy50k": dict(kind="regional", n=50_000, P=10, k=1000, g=1.0, ou=(0.6, 0.2, 10.0), seeds=3),
}


def _network(name):
    d = NETWORKS[name]
    if d["kind"] == "uniform":
        net = nw.make_uniform_block(d["n"], d["k"], seed=0)
        return dict(net=net, spec=None, pop_of=np.zeros(d["n"], np.int32), sizes=np.array([d["n"]]), ou=d["ou"])
    spec = nw.structured_spec(d["n"], d["P"], d["k"], 1, g_scale=np.full((d["P"], 4), d["g"]))
    return dict(net=cc.structured_edges(spec), spec=spec, pop_of=np.repeat(np.arange(d["P"]), spec.pop_sizes).astype(np.int32),
                sizes=np.asarray(spec.pop_sizes), ou=d["ou"])


def _oracle_stats(nd, chunks):
    o = cc.COracleEvents(nd["net"], nd["pop_of"], warm=WARM, ou=nd["ou"])
    for z, _ in chunks:
        o.run(z)
    rates = o.pop_spikes / nd["sizes"] / ((STEPS - WARM) * DT * 1e-3)
    return rates, o.isi_cv()


_CACHE = {}


def _reference(name):
    """Network, oracle statistics for the paired stream (seed 0) and for
    `seeds` independent streams (seed-to-seed spread)."""
    if name not in _CACHE:
        _CACHE.clear()          # one network's data at a time
        nd = _network(name)
        n = nd["pop_of"].shape[0]
        nd["noise"] = list(lo.torch_noise_chunks(0, n, STEPS, CHUNK))   # the paired stream, kept for the engine
        per_seed = [_oracle_stats(nd, nd["noise"] if s == 0 else lo.torch_noise_chunks(s, n, STEPS, CHUNK))
                    for s in range(NETWORKS[name]["seeds"])]
        nd["paired"] = per_seed[0]
        rates = np.array([r for r, _ in per_seed])
        cvs = np.array([c for _, c in per_seed])
        pooled = (rates * nd["sizes"]).sum(1) / nd["sizes"].sum()
        nd["unpaired"] = dict(rates=rates.mean(0), rates_sd=rates.std(0, ddof=1), cv=cvs.mean(), cv_sd=cvs.std(ddof=1),
                              pooled=pooled.mean(), pooled_sd=pooled.std(ddof=1))
        _CACHE[name] = nd
    return _CACHE[name]


def _engine(nd, wt, seed):
    opts = dict(weight_type=wt, seed=seed, ou=nd["ou"])
    if nd["spec"] is None:
        return E.Engine.from_arrays(nd["net"], **opts)
    return E.Engine.structured(nd["spec"], **opts)


def _gpu_stats(nd, wt, variant, paired, seed=1234):
    with _engine(nd, wt, seed) as eng:
        if variant != "auto":
            kind, param = variant.split(":")
            eng.set_push_variant({"reg": E.PUSH_REG, "local": E.PUSH_LOCAL}[kind], int(param))
        isi = IsiMoments(eng.n, WARM)
        counts = []
        for c, t0 in enumerate(range(0, STEPS, CHUNK)):
            if paired:
                eng.set_noise_injected(nd["noise"][c][0])
            r = eng.run(CHUNK, freq=True, record_spikes=True, syn_mode=E.SYN_PUSH)
            counts.append(r.freqs.copy())
            isi.add(r.spikes, t0)
        info = eng.info()
    rates = population_rates(np.concatenate(counts), nd["sizes"], DT, WARM)
    return rates, isi.cv(), f"{['reg', 'tma', 'local'][info.push_kind]}:{info.push_param}"


VARIANTS = [(E.W_F32, "auto"), (E.W_F32, "local:2008"), (E.W_F32, "reg:8"), (E.W_BF16, "auto"), (E.W_BF16, "local:2016")]
# network-major, so each network's oracle runs once
CASES = [
    c for name in NETWORKS for c in ([(name, "paired", wt, v) for wt, v in VARIANTS] +
                                     [(name, "philox", wt, "auto") for wt in (E.W_F32, E.W_BF16)])]


def _wname(wt):
    return "f32" if wt == E.W_F32 else "bf16"


def _check_paired(nd, name, wt, variant):
    r_ref, cv_ref = nd["paired"]
    rates, cv, used = _gpu_stats(nd, wt, variant, paired=True)
    rel = np.abs(rates - r_ref) / r_ref
    cv_rel = abs(cv - cv_ref) / cv_ref
    print("STATS " + json.dumps(dict(test="paired", net=name, weights=_wname(wt), variant=variant, used=used,
                                     rate_hz=float((rates * nd["sizes"]).sum() / nd["sizes"].sum()),
                                     rate_rel_max=float(rel.max()), cv=cv, cv_ref=cv_ref, cv_rel=cv_rel)))
    assert r_ref.min() > 1.0
    assert rel.max() <= RATE_BAR, (rates, r_ref)
    assert cv_rel <= CV_BAR, (cv, cv_ref)


def _check_philox(nd, name, wt):
    u = nd["unpaired"]
    rates, cv, used = _gpu_stats(nd, wt, "auto", paired=False)
    pooled = float((rates * nd["sizes"]).sum() / nd["sizes"].sum())
    pooled_bar = max(RATE_BAR, 4 * u["pooled_sd"] / u["pooled"])
    rate_bar = np.maximum(RATE_BAR, 4 * u["rates_sd"] / u["rates"])
    cv_bar = max(CV_BAR, 4 * u["cv_sd"] / u["cv"])
    rel = np.abs(rates - u["rates"]) / u["rates"]
    print("STATS " + json.dumps(dict(test="philox", net=name, weights=_wname(wt), used=used, pooled_hz=pooled,
                                     pooled_ref=u["pooled"], pooled_rel=abs(pooled - u["pooled"]) / u["pooled"],
                                     pooled_bar=pooled_bar, rate_rel_max=float(rel.max()),
                                     rate_bar_max=float(rate_bar.max()), cv=cv, cv_ref=u["cv"],
                                     cv_rel=abs(cv - u["cv"]) / u["cv"], cv_bar=cv_bar)))
    assert abs(pooled - u["pooled"]) <= pooled_bar * u["pooled"]
    assert np.all(rel <= rate_bar), (rates, u["rates"], rate_bar)
    assert abs(cv - u["cv"]) <= cv_bar * u["cv"], (cv, u["cv"], cv_bar)


@pytest.mark.parametrize("name,mode,wt,variant", CASES, ids=[f"{n}-{m}-{_wname(w)}-{v}" for n, m, w, v in CASES])
def test_statistical_bar(gpu, name, mode, wt, variant):
    nd = _reference(name)
    if mode == "paired":
        _check_paired(nd, name, wt, variant)
    else:
        _check_philox(nd, name, wt)
