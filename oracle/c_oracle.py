"""ctypes front of the C oracle (dtb_oracle.c) -- TEST INFRASTRUCTURE ONLY.

``build_oracle()`` compiles ``oracle/_build/liboracle.so`` with gcc
(-O3 -fopenmp -ffp-contract=off: no fused multiply-add, so float32 results
match the numpy oracle bit for bit).  ``COracle`` mirrors ``lif_oracle.LifOracle``
(same constants, same state) but runs the step loop in C over OpenMP threads;
it is the timed CPU port of the reference model and a fast checker for large
networks.  ``structured_edges`` replays the engine's regional-network edge
stream on the host.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from . import lif_oracle as lo

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIB_PATH = os.path.join(BUILD, "liboracle.so")
SRC = os.path.join(HERE, "dtb_oracle.c")


def build_oracle(force=False):
    if not force and os.path.exists(LIB_PATH) and os.path.getmtime(LIB_PATH) >= os.path.getmtime(SRC):
        return LIB_PATH
    os.makedirs(BUILD, exist_ok=True)
    cmd = ["gcc", "-O3", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
           "-o", LIB_PATH + ".tmp", SRC, "-lm"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    os.replace(LIB_PATH + ".tmp", LIB_PATH)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build_oracle())
        _lib.oracle_run.restype = C.c_int64
        _lib.oracle_run.argtypes = [C.c_void_p, C.c_int32, C.c_float, C.c_void_p, C.c_void_p, C.c_int,
                                    C.c_void_p, C.c_void_p]
        _lib.oracle_structured_edges.restype = None
        _lib.oracle_structured_edges.argtypes = [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64,
                                                 C.c_int32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p,
                                                 C.c_void_p]
        _lib.oracle_threads.restype = C.c_int32
        _lib.oracle_run_f64.restype = C.c_int64
        _lib.oracle_run_f64.argtypes = [C.c_void_p, C.c_int32, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_int32, C.c_int32]
        _lib.oracle_run_events.restype = C.c_int64
        _lib.oracle_run_events.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_float, C.c_void_p, C.c_void_p,
                                           C.c_int, C.c_void_p]
    return _lib


class _Net(C.Structure):
    _fields_ = [("n", C.c_int32)] + [(f, C.c_void_p) for f in (
        "in_ptr", "in_pre", "in_kind", "w0", "w1", "dtC", "neg_gL", "V_L", "V_th", "V_reset", "T_ref", "I_ext",
        "noise_rate", "g", "Vu", "decay", "ou_mean", "ou_f1", "ou_f2s", "V", "i_bg", "t_last", "J", "I_syn", "t",
        "active", "prop")]


def structured_edges(spec):
    """Host replay of the device edge stream (same result as csr_oracle.structured_edges)."""
    n, k = spec.n, spec.in_degree
    s = n * k
    pre = np.empty(s, np.uint32)
    kind = np.empty(s, np.uint8)
    w0 = np.empty(s, np.float32)
    w1 = np.empty(s, np.float32)
    off = spec.pop_offsets.astype(np.uint32)
    exc = np.ascontiguousarray(spec.pop_exc, np.uint32)
    cdf = np.ascontiguousarray(spec.src_cdf, np.uint64)
    lib().oracle_structured_edges(spec.n_pops, off.ctypes.data, exc.ctypes.data, cdf.ctypes.data, spec.seed,
                                  int(spec.dyadic_weights), k, pre.ctypes.data, kind.ctypes.data,
                                  w0.ctypes.data, w1.ctypes.data)
    return dict(property=spec.property_matrix(), input_block_idx=np.zeros(s, np.int16), input_neuron_idx=pre,
                output_neuron_idx=np.repeat(np.arange(n, dtype=np.uint32), k),
                input_channel_offset=(kind * 2).astype(np.uint8), weight=np.stack([w0, w1], axis=1))


class COracle:
    """C-speed twin of ``lif_oracle.LifOracle`` (float32 only)."""

    def __init__(self, net, dt=0.1, ou=(0.6, 0.2, 10.0), prop_mode=lo.PROP_THRESHOLD):
        ref = lo.LifOracle(dict(property=net["property"], input_neuron_idx=np.zeros(0, np.uint32),
                                output_neuron_idx=np.zeros(0, np.uint32),
                                input_channel_offset=np.zeros(0, np.uint8), weight=np.zeros((0, 2), np.float32)),
                           dt=dt, ou=ou, prop_mode=prop_mode)
        self.ref = ref
        self.n = n = ref.n
        self.dt = dt
        self.prop_mode = prop_mode
        post = np.asarray(net["output_neuron_idx"], np.int64)
        order = np.argsort(post, kind="stable")
        self.in_ptr = np.concatenate([[0], np.cumsum(np.bincount(post, minlength=n))]).astype(np.int64)
        self.in_pre = np.ascontiguousarray(np.asarray(net["input_neuron_idx"], np.uint32)[order])
        self.in_kind = np.ascontiguousarray((np.asarray(net["input_channel_offset"]) != 0)[order].astype(np.uint8))
        w = np.asarray(net["weight"], np.float32)[order]
        self.w0 = np.ascontiguousarray(w[:, 0])
        self.w1 = np.ascontiguousarray(w[:, 1])
        f32 = lambda a: np.ascontiguousarray(np.broadcast_to(a, (n,)), np.float32)  # noqa: E731
        self.consts = dict(dtC=f32(ref.dtC), neg_gL=f32(ref.neg_gL), V_L=f32(ref.V_L), V_th=f32(ref.V_th),
                           V_reset=f32(ref.V_reset), T_ref=f32(ref.T_ref), I_ext=f32(ref.i_ext),
                           noise_rate=f32(ref.noise_rate), g=np.ascontiguousarray(ref.g_u, np.float32),
                           Vu=np.ascontiguousarray(ref.V_u, np.float32),
                           decay=np.ascontiguousarray(ref.decay, np.float32), ou_mean=f32(ref.ou_mean),
                           ou_f1=f32(ref.ou_f1), ou_f2s=f32(ref.ou_f2s))
        self.V = f32(ref.V).copy()
        self.i_bg = f32(ref.i_bg).copy()
        self.t_last = f32(ref.t_last).copy()
        self.J = np.zeros((4, n), np.float32)
        self.I_syn = np.zeros(n, np.float32)
        self.t = np.zeros(1, np.float32)
        self._active = np.zeros(n, np.uint8)
        self._prop = np.zeros(n, np.uint8)
        self._s = _Net(n, *(a.ctypes.data for a in (
            self.in_ptr, self.in_pre, self.in_kind, self.w0, self.w1, self.consts["dtC"], self.consts["neg_gL"],
            self.consts["V_L"], self.consts["V_th"], self.consts["V_reset"], self.consts["T_ref"],
            self.consts["I_ext"], self.consts["noise_rate"], self.consts["g"], self.consts["Vu"],
            self.consts["decay"], self.consts["ou_mean"], self.consts["ou_f1"], self.consts["ou_f2s"], self.V,
            self.i_bg, self.t_last, self.J, self.I_syn, self.t, self._active, self._prop)))

    def run(self, z, u=None, record=True):
        """Run z.shape[0] steps; returns (spikes [steps, n] bool or None, counts [steps], events)."""
        z = np.ascontiguousarray(z, np.float32)
        steps = z.shape[0]
        u = None if u is None else np.ascontiguousarray(u, np.float32)
        sp = np.zeros((steps, self.n), np.uint8) if record else None
        counts = np.zeros(steps, np.int64)
        ev = lib().oracle_run(C.byref(self._s), steps, self.dt, z.ctypes.data, None if u is None else u.ctypes.data,
                              self.prop_mode, None if sp is None else sp.ctypes.data, counts.ctypes.data)
        return (None if sp is None else sp.astype(bool)), counts, int(ev)


class _Net64(C.Structure):
    _fields_ = [("n", C.c_int32)] + [(f, C.c_void_p) for f in (
        "in_ptr", "in_pre", "in_kind", "w0", "w1", "dtC", "neg_gL", "V_L", "V_th", "V_reset", "T_ref", "I_ext",
        "g", "Vu", "decay", "ou_mean", "ou_f1", "ou_f2s", "V", "i_bg", "t_last", "J", "I_syn", "t", "active")]


class COracle64:
    """The FP64 restatement (block_new in float64): constants from
    ``LifOracle(dtype=float64)``, state and arithmetic in double, threshold
    propagation.  The normal draws are the float32 stream every run shares."""

    def __init__(self, net, dt=0.1, ou=(0.6, 0.2, 10.0)):
        ref = lo.LifOracle(dict(property=net["property"], input_neuron_idx=np.zeros(0, np.uint32),
                                output_neuron_idx=np.zeros(0, np.uint32),
                                input_channel_offset=np.zeros(0, np.uint8), weight=np.zeros((0, 2), np.float32)),
                           dt=dt, ou=ou, dtype=np.float64)
        self.n = n = ref.n
        self.dt = dt
        post = np.asarray(net["output_neuron_idx"], np.int64)
        order = np.argsort(post, kind="stable")
        self.in_ptr = np.concatenate([[0], np.cumsum(np.bincount(post, minlength=n))]).astype(np.int64)
        self.in_pre = np.ascontiguousarray(np.asarray(net["input_neuron_idx"], np.uint32)[order])
        self.in_kind = np.ascontiguousarray((np.asarray(net["input_channel_offset"]) != 0)[order].astype(np.uint8))
        w = np.asarray(net["weight"], np.float32)[order]
        self.w0 = np.ascontiguousarray(w[:, 0], np.float64)
        self.w1 = np.ascontiguousarray(w[:, 1], np.float64)
        f64 = lambda a: np.ascontiguousarray(np.broadcast_to(a, (n,)), np.float64)  # noqa: E731
        self.consts = [f64(ref.dtC), f64(ref.neg_gL), f64(ref.V_L), f64(ref.V_th), f64(ref.V_reset), f64(ref.T_ref),
                       f64(ref.i_ext), np.ascontiguousarray(ref.g_u, np.float64),
                       np.ascontiguousarray(ref.V_u, np.float64), np.ascontiguousarray(ref.decay, np.float64),
                       f64(ref.ou_mean), f64(ref.ou_f1), f64(ref.ou_f2s)]
        self.V = f64(ref.V).copy()
        self.i_bg = f64(ref.i_bg).copy()
        self.t_last = f64(ref.t_last).copy()
        self.J = np.zeros((4, n), np.float64)
        self.I_syn = np.zeros(n, np.float64)
        self.t = np.zeros(1, np.float64)
        self._active = np.zeros(n, np.uint8)
        self._s = _Net64(n, *(a.ctypes.data for a in (
            [self.in_ptr, self.in_pre, self.in_kind, self.w0, self.w1] + self.consts +
            [self.V, self.i_bg, self.t_last, self.J, self.I_syn, self.t, self._active])))

    def run(self, z, record=True, n_v=0, clock32=False):
        """Run z.shape[0] steps; returns (spikes [steps, n] bool or None, counts [steps], events,
        V of the first n_v neurons after every step as float32 [steps, n_v]).  clock32 keeps the
        clock in float32 (block_new's time) and everything else in double."""
        z = np.ascontiguousarray(z, np.float32)
        steps = z.shape[0]
        sp = np.zeros((steps, self.n), np.uint8) if record else None
        counts = np.zeros(steps, np.int64)
        vt = np.zeros((steps, n_v), np.float32) if n_v else None
        ev = lib().oracle_run_f64(C.byref(self._s), steps, self.dt, z.ctypes.data,
                                  None if sp is None else sp.ctypes.data, counts.ctypes.data,
                                  None if vt is None else vt.ctypes.data, n_v, int(clock32))
        return (None if sp is None else sp.astype(bool)), counts, int(ev), vt


class _Events(C.Structure):
    _fields_ = [("out_ptr", C.c_void_p), ("out_post", C.c_void_p), ("out_kind", C.c_void_p), ("ow0", C.c_void_p),
                ("ow1", C.c_void_p), ("pop_of", C.c_void_p), ("n_pops", C.c_int32), ("step0", C.c_int64),
                ("warm", C.c_int64), ("pop_spikes", C.c_void_p), ("last_spike", C.c_void_p), ("isi", C.c_void_p),
                ("acc", C.c_void_p), ("list", C.c_void_p)]


class COracleEvents(COracle):
    """``COracle`` with the event-driven step (``oracle_run_events``): the same
    float32 results, O(events) per step, plus running population spike counts and
    pooled inter-spike-interval moments from step ``warm`` on -- the long
    statistical runs of the firing-rate / ISI-CV checks."""

    def __init__(self, net, pop_of, warm=0, **kw):
        super().__init__(net, **kw)
        n = self.n
        pre = np.asarray(net["input_neuron_idx"], np.uint32)
        post = np.asarray(net["output_neuron_idx"], np.uint32)
        if post.size and np.all(post[1:] >= post[:-1]):
            order = np.argsort(pre, kind="stable")          # post-major input: rows ascend by target
        else:
            order = np.lexsort((post, pre))
        self.out_ptr = np.concatenate([[0], np.cumsum(np.bincount(pre, minlength=n))]).astype(np.int64)
        self.out_post = np.ascontiguousarray(post[order])
        self.out_kind = np.ascontiguousarray((np.asarray(net["input_channel_offset"]) != 0)[order].astype(np.uint8))
        w = np.asarray(net["weight"], np.float32)
        self.ow0 = np.ascontiguousarray(w[order, 0])
        self.ow1 = np.ascontiguousarray(w[order, 1])
        self.pop_of = np.ascontiguousarray(pop_of, np.int32)
        self.n_pops = int(self.pop_of.max()) + 1 if n else 0
        self.pop_spikes = np.zeros(self.n_pops, np.int64)
        self.last_spike = np.full(n, -1, np.int64)
        self.isi = np.zeros(3, np.float64)
        self._acc = np.zeros(4 * n, np.float64)
        self._list = np.zeros(max(n, 1), np.uint32)
        self._ev = _Events(self.out_ptr.ctypes.data, self.out_post.ctypes.data, self.out_kind.ctypes.data,
                           self.ow0.ctypes.data, self.ow1.ctypes.data, self.pop_of.ctypes.data, self.n_pops, 0,
                           int(warm), self.pop_spikes.ctypes.data, self.last_spike.ctypes.data,
                           self.isi.ctypes.data, self._acc.ctypes.data, self._list.ctypes.data)

    def run(self, z, u=None, record=False):
        """Run z.shape[0] steps; returns (None, counts [steps], events).  Statistics
        accumulate in pop_spikes / isi across calls."""
        if record:
            raise ValueError("the event-driven oracle keeps running statistics, not rasters")
        z = np.ascontiguousarray(z, np.float32)
        steps = z.shape[0]
        u = None if u is None else np.ascontiguousarray(u, np.float32)
        counts = np.zeros(steps, np.int64)
        ev = lib().oracle_run_events(C.byref(self._s), C.byref(self._ev), steps, self.dt, z.ctypes.data,
                                     None if u is None else u.ctypes.data, self.prop_mode, counts.ctypes.data)
        return None, counts, int(ev)

    def isi_cv(self):
        c, s1, s2 = self.isi
        if c < 2:
            return float("nan")
        mean = s1 / c
        return float(np.sqrt(max(s2 / c - mean * mean, 0.0)) / mean)
