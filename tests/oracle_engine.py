"""A CPU stand-in for ``engine.Engine`` built on the numpy oracle -- TEST
INFRASTRUCTURE ONLY.  It has the methods server.py calls, so the gRPC front can be
driven by the reference's own client (python/dist_blockwrapper.py) on a machine
without a GPU; a second instance with the same seed gives the results a direct
call would, to check every answer the client decodes.

The step is oracle/lif_oracle.LifOracle (models/block_new.py's equations), the OU
normal draws come from a numpy generator seeded by ``seed``, the property updates
follow the C-ABI's rules (dtb_update_props / update_prop_cols / update_gamma /
set_ou: PropType ids of protos/snn.proto:94-115 mapped to the property columns of
python/make_block.py:426-464).
"""
from __future__ import annotations

import types

import numpy as np

from dtb_b200 import engine as E
from oracle import lif_oracle as lo

# snn.proto PropType -> column of the [N, 22] property matrix
PROP_COL = {0: 2, 1: 4, 2: 5, 3: 6, 4: 7, 5: 8, 6: 9, 7: 10, 8: 11, 9: 12, 10: 13, 11: 14, 12: 15, 13: 16,
            14: 17, 15: 18, 16: 19, 17: 20, 18: 21, 19: 0}


class OracleEngine:
    def __init__(self, net, dt=0.1, weight_type=E.W_F32, seed=0, push=True, pull=False):
        self.prop = np.asarray(net["property"], np.float32).copy()
        self.o = lo.LifOracle(dict(net, weight=np.asarray(net["weight"], np.float32)), dt=dt)
        self.n = self.prop.shape[0]
        col = self.prop[:, 3]
        starts = np.concatenate([[0], np.nonzero(col[1:] != col[:-1])[0] + 1])
        self.pop_of = np.repeat(np.arange(starts.size), np.diff(np.concatenate([starts, [self.n]])))
        self.pop_ids = col[starts].astype(np.uint32)
        self.pop_sizes = np.bincount(self.pop_of).astype(np.uint32)
        self.n_pops = int(starts.size)
        self.keep = self.prop[:, 1] == 0
        self.rng = np.random.default_rng(seed)
        self.gamma_rng = np.random.default_rng(seed + 1)
        self.samples = np.zeros(0, np.int64)
        self.ou_set = np.zeros(self.n_pops, bool)

    def info(self):
        return types.SimpleNamespace(device_bytes=0, n_neurons=self.n, n_pops=self.n_pops)

    def close(self):
        pass

    def _pop_mean(self, x):
        w = self.keep.astype(np.float64)
        return (np.bincount(self.pop_of, weights=x.astype(np.float64) * w, minlength=self.n_pops) /
                np.maximum(np.bincount(self.pop_of, weights=w, minlength=self.n_pops), 1)).astype(np.float32)

    def run(self, iters, use_ou=True, freq=True, vmean=False, syn_mode=E.SYN_PUSH, sample_spike=False, sample_v=False,
            sample_iou=False, imean=False, receptor_imean=False, sample_isyn=False, t_steps=1, **_):
        if not use_ou or t_steps != 1:
            raise E.DtbError(E.UNSUPPORTED, "the oracle stand-in runs the OU background, one substep")
        P, S = self.n_pops, self.samples
        out = dict(freqs=np.zeros((iters, P), np.int32), vmeans=np.zeros((iters, P), np.float32),
                   imeans=np.zeros((iters, P), np.float32), receptor_imeans=np.zeros((iters, 4, P), np.float32),
                   sample_spike=np.zeros((iters, S.size), np.uint8), sample_v=np.zeros((iters, S.size), np.float32),
                   sample_iou=np.zeros((iters, S.size), np.float32), sample_isyn=np.zeros((iters, S.size), np.float32))
        for s in range(iters):
            active, _ = self.o.step(self.rng.standard_normal(self.n, dtype=np.float32))
            out["freqs"][s] = np.bincount(self.pop_of, weights=active & self.keep, minlength=P)
            out["vmeans"][s] = self._pop_mean(self.o.V)
            out["imeans"][s] = self._pop_mean(self.o.I_syn)
            for c in range(4):
                out["receptor_imeans"][s, c] = self._pop_mean(self.o.I_u[c])
            out["sample_spike"][s] = active[S]
            out["sample_v"][s] = self.o.V[S]
            out["sample_iou"][s] = self.o.i_bg[S]
            out["sample_isyn"][s] = self.o.I_syn[S]
        pick = lambda k, on: out[k] if on else None  # noqa: E731
        return E.RunResult(pick("freqs", freq), pick("vmeans", vmean), None, 0, 0.0, (0.0,) * 4, 0,
                           pick("sample_spike", sample_spike), pick("sample_v", sample_v),
                           pick("sample_iou", sample_iou), pick("imeans", imean),
                           pick("receptor_imeans", receptor_imean), pick("sample_isyn", sample_isyn))

    # ---- property surface (the C-ABI's rules)
    def _refresh(self):
        self.o.set_property(self.prop)

    def update_props(self, nid, pid, val):
        for i, p, v in zip(np.asarray(nid), np.asarray(pid), np.asarray(val, np.float32)):
            if i < self.n and int(p) in PROP_COL:
                self.prop[i, PROP_COL[int(p)]] = v
        self._refresh()

    def update_prop_cols(self, pid, pops, val, assign=False):
        for p, g, v in zip(np.asarray(pid), np.asarray(pops), np.asarray(val, np.float32)):
            m = self.pop_of == int(np.nonzero(self.pop_ids == g)[0][0])
            c = PROP_COL[int(p)]
            self.prop[m, c] = v if assign else self.prop[m, c] * v
        self._refresh()

    def update_gamma(self, pid, pops, alpha, beta):
        for p, g, a, b in zip(np.asarray(pid), np.asarray(pops), np.asarray(alpha), np.asarray(beta)):
            m = self.pop_of == int(np.nonzero(self.pop_ids == g)[0][0])
            self.prop[m, PROP_COL[int(p)]] = (self.gamma_rng.gamma(float(a), size=int(m.sum())) / float(b)).astype(np.float32)
        self._refresh()

    def set_ou(self, pops, mean, sigma, tau):
        for g, mu, sd, ta in zip(np.asarray(pops), np.asarray(mean), np.asarray(sigma), np.asarray(tau)):
            k = int(np.nonzero(self.pop_ids == g)[0][0])
            m = self.pop_of == k
            self.o.set_ou(np.float32(mu), np.float32(sd), np.float32(ta), mask=m)
            if not self.ou_set[k]:
                self.o.i_bg[m] = np.float32(mu)     # the first configuration resets the current to the mean
                self.ou_set[k] = True

    def set_samples(self, ids):
        self.samples = np.asarray(ids, np.int64)
