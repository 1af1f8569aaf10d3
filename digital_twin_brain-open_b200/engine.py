"""ctypes binding of ``include/dtb_b200.h`` -- the host-side mirror of the reference's
block engine (``dtb::BrainBlock``, include/block.hpp:21-889) as driven by the
``snn.proto`` service.

Every call goes to the CUDA library ``libdtb_b200.so`` built in-tree; there is no
CPU fallback: if the library is missing, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdtb_b200.so")

# status codes (dtb_status)
OK, INVALID_PARAMETER, UNSET_SAMPLE_FAILURE, UNSUPPORTED, NOT_ENABLE_METRIC, INVALID_NETWORK = 0, 1, 2, 3, 4, 5
OUT_OF_MEMORY, CUDA_ERROR, DEVICE_FAULT, IO_ERROR, NO_DEVICE = 16, 17, 18, 19, 20

W_F32, W_BF16, W_F16, W_U8, W_F64 = 0, 1, 2, 3, 4
PROP_THRESHOLD, PROP_NOISE, PROP_OR = 0, 1, 2
SYN_PUSH, SYN_PUSH_EXACT, SYN_PULL, SYN_PUSH_FIXED = 0, 1, 2, 3
PUSH_REG, PUSH_TMA, PUSH_LOCAL = 0, 1, 2
NOISE_PHILOX, NOISE_INJECTED = 0, 1
RUN_USE_OU, RUN_FREQ, RUN_VMEAN, RUN_RECORD_SPIKES, RUN_TIME_KERNELS = 1, 2, 4, 8, 16
RUN_SAMPLE_SPIKE, RUN_SAMPLE_V, RUN_SAMPLE_IOU = 32, 64, 128
RUN_IMEAN, RUN_RECEPTOR_IMEAN, RUN_SAMPLE_ISYN = 256, 512, 1024
STATE_V, STATE_J, STATE_I_OU, STATE_T_LAST = 0, 1, 2, 3

# snn.proto PropType
PROP_IDS = dict(EXT_STIMULI_I=0, MEMBRANE_C=1, REF_T=2, LEAKAGE_G=3, LEAKAGE_V=4, THRESHOLD_V=5, RESET_V=6,
                CONDUCT_G_AMPA=7, CONDUCT_G_NMDA=8, CONDUCT_G_GABAa=9, CONDUCT_G_GABAb=10,
                MEMBRANE_V_AMPA=11, MEMBRANE_V_NMDA=12, MEMBRANE_V_GABAa=13, MEMBRANE_V_GABAb=14,
                TAO_AMPA=15, TAO_NMDA=16, TAO_GABAa=17, TAO_GABAb=18, NOISE_RATE=19)


class DtbError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{status_string(status)}: {message}")
        self.status = status


class Options(C.Structure):
    _fields_ = [("dt", C.c_float), ("weight_type", C.c_uint32), ("seed", C.c_uint64),
                ("build_push", C.c_uint32), ("build_pull", C.c_uint32),
                ("ou_mean", C.c_float), ("ou_sigma", C.c_float), ("ou_tau", C.c_float),
                ("reserved", C.c_uint32 * 8)]


class NetworkArrays(C.Structure):
    _fields_ = [("n_neurons", C.c_uint32), ("property", C.c_void_p), ("n_edges", C.c_uint64),
                ("input_block_idx", C.c_void_p), ("input_neuron_idx", C.c_void_p),
                ("output_neuron_idx", C.c_void_p), ("input_channel_offset", C.c_void_p),
                ("weight", C.c_void_p), ("weight_type", C.c_uint32)]


class StructuredSpecC(C.Structure):
    _fields_ = [("n_pops", C.c_uint32), ("pop_sizes", C.c_void_p), ("pop_exc", C.c_void_p),
                ("src_cdf", C.c_void_p), ("pop_property", C.c_void_p), ("pop_id_base", C.c_uint32),
                ("in_degree", C.c_uint32), ("seed", C.c_uint64), ("dyadic_weights", C.c_uint32)]


class EngineInfo(C.Structure):
    _fields_ = [("n_neurons", C.c_uint32), ("n_pops", C.c_uint32), ("n_edges", C.c_uint64),
                ("device_bytes", C.c_uint64), ("step", C.c_uint64), ("t", C.c_float),
                ("weight_type", C.c_uint32), ("has_push", C.c_uint32), ("has_pull", C.c_uint32),
                ("per_neuron_params", C.c_uint32), ("push_kind", C.c_uint32), ("push_param", C.c_uint32),
                ("push_tuned_ms", C.c_float), ("local_windows", C.c_uint32), ("fixed_shift", C.c_uint32),
                ("graph_launches", C.c_uint32)]


class RunRequest(C.Structure):
    _fields_ = [("iters", C.c_uint32), ("flags", C.c_uint32), ("prop_mode", C.c_uint32),
                ("syn_mode", C.c_uint32), ("t_steps", C.c_uint32), ("reserved", C.c_uint32 * 3)]


class RunOutput(C.Structure):
    _fields_ = [("freqs", C.c_void_p), ("vmeans", C.c_void_p), ("spike_bits", C.c_void_p),
                ("events", C.c_uint64), ("device_ms", C.c_double), ("kernel_ms", C.c_double * 4),
                ("launches", C.c_uint32), ("reserved", C.c_uint32), ("sample_spike", C.c_void_p),
                ("sample_v", C.c_void_p), ("sample_iou", C.c_void_p), ("imeans", C.c_void_p),
                ("receptor_imeans", C.c_void_p), ("sample_isyn", C.c_void_p)]


_P = C.c_void_p
_U32 = C.c_uint32
_I32 = C.c_int32
SIGNATURES = {
    "dtb_abi_version": (_I32, []),
    "dtb_engine_version": (_I32, []),
    "dtb_status_string": (C.c_char_p, [_I32]),
    "dtb_last_error": (C.c_char_p, []),
    "dtb_default_options": (None, [_P]),
    "dtb_create": (_I32, [_P, _P, C.POINTER(C.c_void_p)]),
    "dtb_create_structured": (_I32, [_P, _P, C.POINTER(C.c_void_p)]),
    "dtb_create_from_npz": (_I32, [C.c_char_p, _P, C.POINTER(C.c_void_p)]),
    "dtb_destroy": (_I32, [_P]),
    "dtb_info": (_I32, [_P, _P]),
    "dtb_get_stream": (_I32, [_P, C.POINTER(C.c_void_p)]),
    "dtb_set_push_variant": (_I32, [_P, _I32, _I32]),
    "dtb_set_graph": (_I32, [_P, _I32]),
    "dtb_tuning_report": (_I32, [_P, _P, _P, _P, _P]),
    "dtb_populations": (_I32, [_P, _P, _P]),
    "dtb_update_props": (_I32, [_P, _U32, _P, _P, _P]),
    "dtb_update_prop_cols": (_I32, [_P, _U32, _P, _P, _P, _I32]),
    "dtb_update_gamma": (_I32, [_P, _U32, _P, _P, _P, _P]),
    "dtb_set_ou": (_I32, [_P, _U32, _P, _P, _P, _P]),
    "dtb_read_property": (_I32, [_P, _U32, _P]),
    "dtb_set_noise": (_I32, [_P, _U32, _U32, _P, _P]),
    "dtb_set_samples": (_I32, [_P, _U32, _P]),
    "dtb_run": (_I32, [_P, _P, _P]),
    "dtb_read_state": (_I32, [_P, _I32, _P]),
    "dtb_write_state": (_I32, [_P, _I32, _P]),
    "dtb_read_out_csr": (_I32, [_P, _P, _P, _P, _P, _P, _P, _P]),
    "dtb_state_size": (_I32, [_P, _P]),
    "dtb_save_state": (_I32, [_P, _P, C.c_uint64]),
    "dtb_load_state": (_I32, [_P, _P, C.c_uint64]),
    "dtb_build_out_csr_host": (_I32, [_U32, C.c_uint64, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "dtb_compact_spikes": (_I32, [_P, _U32, _P, _P, _P]),
    "dtb_batch_create": (_I32, [_P, _U32, C.POINTER(C.c_void_p)]),
    "dtb_batch_destroy": (_I32, [_P]),
    "dtb_batch_run": (_I32, [_P, _P, _P]),
    "dtb_batch_set_graph": (_I32, [_P, _I32]),
    "dtb_batch_set_push_variant": (_I32, [_P, _I32, _I32]),
    "dtb_batch_info": (_I32, [_P, _P, _P, _P, _P]),
    "dtb_compact_spikes_noalloc": (_I32, [_P, _U32, _P, _P, _P]),
    "dtb_bold_default_params": (None, [_P]),
    "dtb_bold_run": (_I32, [_P, _U32, _U32, _P, _P, _P, _P]),
    "dtb_da_filter": (_I32, [_U32, _U32, _U32, _P, _P, _P, C.c_double, C.c_double, _P, _P]),
    "dtb_server_default_options": (None, [_P]),
    "dtb_server_create": (_I32, [_P, C.POINTER(C.c_void_p)]),
    "dtb_server_destroy": (_I32, [_P]),
    "dtb_server_add_structured": (_I32, [_P, _P, _P, _P]),
    "dtb_server_add_npz": (_I32, [_P, C.c_char_p, _P, _P]),
    "dtb_server_play": (_I32, [_P, _U32, _P, _U32]),
    "dtb_server_info": (_I32, [_P, _P]),
    "dtb_server_start": (_I32, [_P, _U32]),
    "dtb_server_submit": (_I32, [_P, _P, C.POINTER(C.c_uint64)]),
    "dtb_server_poll": (_I32, [_P, C.c_uint64, _U32, C.POINTER(C.c_int32)]),
    "dtb_server_stop": (_I32, [_P]),
}


def load_library(path=LIB_PATH):
    if not os.path.exists(path):
        raise ImportError(f"libdtb_b200.so not built ({path}); run digital_twin_brain-open_b200/build.py")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


LIB = load_library()


def status_string(status):
    return LIB.dtb_status_string(int(status)).decode()


def _check(status):
    if status != OK:
        raise DtbError(status, LIB.dtb_last_error().decode())


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def default_options(dt=0.1, weight_type=W_F32, seed=0, push=True, pull=False, ou=(0.6, 0.2, 10.0)):
    o = Options()
    LIB.dtb_default_options(C.byref(o))
    o.dt = dt
    o.weight_type = weight_type
    o.seed = seed
    o.build_push = int(push)
    o.build_pull = int(pull)
    o.ou_mean, o.ou_sigma, o.ou_tau = ou
    return o


def build_out_csr_host(n, pre, post, kind):
    """The reference's out-degree CSR built on the host (no GPU): rows, row_ptr, post, kind, perm."""
    pre, post = _u32(pre), _u32(post)
    kind = np.ascontiguousarray(kind, np.uint8)
    s = pre.shape[0]
    rows = np.empty(n, np.uint32)
    row_ptr = np.empty(n + 1, np.uint64)
    post_o = np.empty(s, np.uint32)
    kind_o = np.empty(s, np.uint8)
    perm = np.empty(s, np.uint64)
    nr = C.c_uint32()
    _check(LIB.dtb_build_out_csr_host(n, s, _ptr(pre), _ptr(post), _ptr(kind), C.byref(nr), _ptr(rows),
                                      _ptr(row_ptr), _ptr(post_o), _ptr(kind_o), _ptr(perm)))
    nr = nr.value
    return rows[:nr], row_ptr[:nr + 1], post_o, kind_o, perm


def compact_spikes(d_bits, n, d_indices, d_count, stream=0):
    """Device spike bitmap -> ascending device index list (all pointers are device addresses)."""
    _check(LIB.dtb_compact_spikes(C.c_void_p(d_bits), n, C.c_void_p(d_indices), C.c_void_p(d_count),
                                  C.c_void_p(stream) if stream else None))


class ServerOptions(C.Structure):
    _fields_ = [("hbm_cap_bytes", C.c_uint64), ("slice_steps", C.c_uint32), ("max_batch", C.c_uint32),
                ("syn_mode", C.c_uint32), ("flags", C.c_uint32), ("autotune", C.c_uint32),
                ("reserved", C.c_uint32 * 3)]


class Request(C.Structure):
    _fields_ = [("net", C.c_uint32), ("iters", C.c_uint32), ("arrival_s", C.c_double),
                ("ou_mean", C.c_void_p), ("ou_sigma", C.c_void_p), ("ou_tau", C.c_void_p),
                ("freqs", C.c_void_p), ("start_s", C.c_double), ("finish_s", C.c_double),
                ("events", C.c_uint64), ("status", C.c_int32), ("reserved", C.c_uint32)]


class ServerInfo(C.Structure):
    _fields_ = [("n_nets", C.c_uint32), ("resident", C.c_uint32), ("resident_bytes", C.c_uint64),
                ("evictions", C.c_uint64), ("restores", C.c_uint64), ("slices", C.c_uint64),
                ("batch_members_sum", C.c_uint64)]


SERVE_BATCHED, SERVE_SEQUENTIAL = 0, 1


class BoldParams(C.Structure):
    _fields_ = [(f, C.c_double) for f in ("epsilon", "tao_s", "tao_f", "tao_0", "alpha", "E_0", "V_0", "delta_t")]


def bold_params(**kw):
    """dtb_bold_params with DA_voxel.py's defaults, overridden by keyword."""
    p = BoldParams()
    LIB.dtb_bold_default_params(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, float(v))
    return p


def da_filter(w_hat, bold_y, noise, bold_sigma, rate=0.5, stream=0):
    """DA_voxel.filter on CUDA float32 torch tensors w_hat [E, V, S], bold_y [V], noise [E, V]."""
    import torch
    assert w_hat.is_cuda and w_hat.dtype == torch.float32
    E, V, S = w_hat.shape
    w_hat, bold_y, noise = w_hat.contiguous(), bold_y.contiguous(), noise.contiguous()
    out = torch.empty_like(w_hat)
    _check(LIB.dtb_da_filter(E, V, S, C.c_void_p(w_hat.data_ptr()), C.c_void_p(bold_y.data_ptr()),
                             C.c_void_p(noise.data_ptr()), float(bold_sigma), float(rate), C.c_void_p(out.data_ptr()),
                             C.c_void_p(stream)))
    return out


def bold_run(u, state, params=None, out=True, stream=0):
    """BOLD.run over a window: u, state are CUDA float32 torch tensors ([steps, n], [4, n]:
    s, q, v, f_in, advanced in place); returns the [steps, n] signal (or None)."""
    import torch
    assert u.is_cuda and state.is_cuda and u.dtype == torch.float32 and state.dtype == torch.float32
    steps, n = u.shape
    u = u.contiguous()
    o = torch.empty_like(u) if out else None
    p = params or bold_params()
    _check(LIB.dtb_bold_run(C.byref(p), n, steps, C.c_void_p(u.data_ptr()), C.c_void_p(state.data_ptr()),
                            None if o is None else C.c_void_p(o.data_ptr()), C.c_void_p(stream)))
    return o


@dataclasses.dataclass
class RunResult:
    freqs: np.ndarray | None
    vmeans: np.ndarray | None
    spikes: np.ndarray | None      # bool [iters, n] threshold spikes
    events: int
    device_ms: float
    kernel_ms: tuple = (0.0, 0.0, 0.0, 0.0)   # LIF, push, pull, end-of-run (with time_kernels)
    launches: int = 0
    sample_spike: np.ndarray | None = None   # uint8 [iters, n_samples]
    sample_v: np.ndarray | None = None
    sample_iou: np.ndarray | None = None
    imeans: np.ndarray | None = None             # float [iters, P] mean I_syn at the end of each step
    receptor_imeans: np.ndarray | None = None    # float [iters, 4, P] mean I_AMPA, I_NMDA, I_GABAa, I_GABAb
    sample_isyn: np.ndarray | None = None        # float [iters, n_samples] end-of-step I_syn


class Engine:
    """One network resident in HBM (reference: BrainBlock + snn_run)."""

    def __init__(self, handle):
        self._h = C.c_void_p(handle)
        inf = self.info()
        self.n = inf.n_neurons
        self.n_pops = inf.n_pops
        self.pop_ids, self.pop_sizes = self.populations()

    # ---- construction
    @classmethod
    def from_arrays(cls, net, **opts):
        prop = _f32(net["property"])
        n = prop.shape[0]
        w = np.ascontiguousarray(net["weight"])
        wt = {np.dtype(np.float32): W_F32, np.dtype(np.float64): W_F64, np.dtype(np.float16): W_F16,
              np.dtype(np.uint8): W_U8}[w.dtype]
        pre = _u32(net["input_neuron_idx"])
        post = _u32(net["output_neuron_idx"])
        kind = np.ascontiguousarray(net["input_channel_offset"], np.uint8)
        blk = net.get("input_block_idx")
        blk = None if blk is None else np.ascontiguousarray(blk, np.int16)
        a = NetworkArrays(n, prop.ctypes.data, pre.shape[0], None if blk is None else blk.ctypes.data,
                          pre.ctypes.data, post.ctypes.data, kind.ctypes.data, w.ctypes.data, wt)
        o = default_options(**opts)
        h = C.c_void_p()
        _check(LIB.dtb_create(C.byref(a), C.byref(o), C.byref(h)))
        return cls(h.value)

    @classmethod
    def structured(cls, spec, pop_id_base=0, **opts):
        sizes = _u32(spec.pop_sizes)
        exc = _u32(spec.pop_exc)
        cdf = np.ascontiguousarray(spec.src_cdf, np.uint64)
        prop = np.ascontiguousarray(spec.property_rows(), np.float32)
        s = StructuredSpecC(spec.n_pops, sizes.ctypes.data, exc.ctypes.data, cdf.ctypes.data, prop.ctypes.data,
                            pop_id_base, spec.in_degree, spec.seed, int(spec.dyadic_weights))
        o = default_options(**opts)
        h = C.c_void_p()
        _check(LIB.dtb_create_structured(C.byref(s), C.byref(o), C.byref(h)))
        return cls(h.value)

    @classmethod
    def from_npz(cls, path, **opts):
        o = default_options(**opts)
        h = C.c_void_p()
        _check(LIB.dtb_create_from_npz(os.fsencode(path), C.byref(o), C.byref(h)))
        return cls(h.value)

    def close(self):
        if self._h is not None and self._h.value:
            _check(LIB.dtb_destroy(self._h))
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- queries
    def info(self):
        inf = EngineInfo()
        _check(LIB.dtb_info(self._h, C.byref(inf)))
        return inf

    def set_push_variant(self, kind, param=0):
        """kind 0: register-staged (param 4/8/16, 1016/1008 sub-warp rows), 1: TMA-staged
        (param 256/512), 2: population-local windows (param 8/1016), -1: autotune."""
        _check(LIB.dtb_set_push_variant(self._h, kind, param))

    def set_graph(self, enable):
        """Replay repeated run chunks from captured CUDA graphs (default on)."""
        _check(LIB.dtb_set_graph(self._h, int(enable)))

    def tuning_report(self):
        """[(kind, param, ms)] of the push variants timed by the autotuner."""
        n = C.c_uint32(16)
        k = np.zeros(16, np.int32)
        p = np.zeros(16, np.int32)
        ms = np.zeros(16, np.float32)
        _check(LIB.dtb_tuning_report(self._h, C.byref(n), _ptr(k), _ptr(p), _ptr(ms)))
        return [(int(k[i]), int(p[i]), float(ms[i])) for i in range(min(n.value, 16))]

    def stream(self):
        """The engine's cudaStream_t as an integer handle."""
        s = C.c_void_p()
        _check(LIB.dtb_get_stream(self._h, C.byref(s)))
        return s.value or 0

    def populations(self):
        p = self.info().n_pops
        ids = np.empty(p, np.uint32)
        counts = np.empty(p, np.uint32)
        _check(LIB.dtb_populations(self._h, _ptr(ids), _ptr(counts)))
        return ids, counts

    # ---- property surface
    def update_props(self, neuron_ids, prop_ids, values):
        nid, pid, val = _u32(neuron_ids), _u32(prop_ids), _f32(values)
        _check(LIB.dtb_update_props(self._h, nid.shape[0], _ptr(nid), _ptr(pid), _ptr(val)))

    def update_prop_cols(self, prop_ids, pop_ids, values, assign=False):
        pid, pop, val = _u32(prop_ids), _u32(pop_ids), _f32(values)
        _check(LIB.dtb_update_prop_cols(self._h, pid.shape[0], _ptr(pid), _ptr(pop), _ptr(val), int(assign)))

    def update_gamma(self, prop_ids, pop_ids, alpha, beta):
        pid, pop, a, b = _u32(prop_ids), _u32(pop_ids), _f32(alpha), _f32(beta)
        _check(LIB.dtb_update_gamma(self._h, pid.shape[0], _ptr(pid), _ptr(pop), _ptr(a), _ptr(b)))

    def read_property(self, prop_id):
        """Per-neuron value of property ``prop_id`` (PROP_IDS) as the updates left it."""
        a = np.empty(self.n, np.float32)
        _check(LIB.dtb_read_property(self._h, int(prop_id), _ptr(a)))
        return a

    def set_ou(self, pop_ids, mean, sigma, tau):
        pop, m, s, t = _u32(pop_ids), _f32(mean), _f32(sigma), _f32(tau)
        _check(LIB.dtb_set_ou(self._h, pop.shape[0], _ptr(pop), _ptr(m), _ptr(s), _ptr(t)))

    def set_noise_injected(self, z, u=None):
        z = _f32(z)
        u = None if u is None else _f32(u)
        _check(LIB.dtb_set_noise(self._h, NOISE_INJECTED, z.shape[0], _ptr(z), _ptr(u)))

    def set_samples(self, neuron_ids):
        idx = _u32(neuron_ids)
        _check(LIB.dtb_set_samples(self._h, idx.shape[0], _ptr(idx)))
        self.n_sample_list = int(idx.shape[0])

    def set_noise_philox(self):
        _check(LIB.dtb_set_noise(self._h, NOISE_PHILOX, 0, None, None))

    # ---- stepping
    def run(self, iters, use_ou=True, freq=True, vmean=False, record_spikes=False,
            prop_mode=PROP_THRESHOLD, syn_mode=SYN_PUSH, time_kernels=False, out=None,
            sample_spike=False, sample_v=False, sample_iou=False, imean=False, receptor_imean=False,
            sample_isyn=False, t_steps=1):
        """Advance ``iters`` steps (RunRequest, snn.proto:63-77), each of ``t_steps``
        substeps of dt / t_steps when t_steps > 1.

        ``out`` may pass preallocated (freqs, vmeans) host arrays of shape [iters, P].
        """
        flags = (RUN_USE_OU if use_ou else 0) | (RUN_FREQ if freq else 0) | \
                (RUN_VMEAN if vmean else 0) | (RUN_RECORD_SPIKES if record_spikes else 0) | \
                (RUN_TIME_KERNELS if time_kernels else 0) | (RUN_SAMPLE_SPIKE if sample_spike else 0) | \
                (RUN_SAMPLE_V if sample_v else 0) | (RUN_SAMPLE_IOU if sample_iou else 0) | \
                (RUN_IMEAN if imean else 0) | (RUN_RECEPTOR_IMEAN if receptor_imean else 0) | \
                (RUN_SAMPLE_ISYN if sample_isyn else 0)
        im = np.zeros((iters, self.n_pops), np.float32) if imean else None
        rim = np.zeros((iters, 4, self.n_pops), np.float32) if receptor_imean else None
        ns = getattr(self, "n_sample_list", 0)
        ss = np.zeros((iters, ns), np.uint8) if sample_spike else None
        sv = np.zeros((iters, ns), np.float32) if sample_v else None
        si = np.zeros((iters, ns), np.float32) if sample_iou else None
        sy = np.zeros((iters, ns), np.float32) if sample_isyn else None
        rq = RunRequest(iters, flags, prop_mode, syn_mode, t_steps)
        if out is not None:
            fr, vm = out
        else:
            fr = np.zeros((iters, self.n_pops), np.int32) if freq else None
            vm = np.zeros((iters, self.n_pops), np.float32) if vmean else None
        words = (self.n + 31) // 32
        sb = np.zeros((iters, words), np.uint32) if record_spikes else None
        res = RunOutput(None if fr is None else fr.ctypes.data, None if vm is None else vm.ctypes.data,
                        None if sb is None else sb.ctypes.data, 0, 0.0)
        res.sample_spike = None if ss is None else ss.ctypes.data
        res.sample_v = None if sv is None else sv.ctypes.data
        res.sample_iou = None if si is None else si.ctypes.data
        res.imeans = None if im is None else im.ctypes.data
        res.receptor_imeans = None if rim is None else rim.ctypes.data
        res.sample_isyn = None if sy is None else sy.ctypes.data
        _check(LIB.dtb_run(self._h, C.byref(rq), C.byref(res)))
        spikes = None
        if sb is not None:
            spikes = np.unpackbits(sb.view(np.uint8), axis=1, bitorder="little")[:, :self.n].astype(bool)
        return RunResult(fr, vm, spikes, int(res.events), float(res.device_ms), tuple(res.kernel_ms), int(res.launches),
                         ss, sv, si, im, rim, sy)

    # ---- state
    def read_state(self, which):
        shape = (self.n, 4) if which == STATE_J else (self.n,)
        a = np.empty(shape, np.float32)
        _check(LIB.dtb_read_state(self._h, which, _ptr(a)))
        return a

    def write_state(self, which, a):
        a = _f32(a)
        _check(LIB.dtb_write_state(self._h, which, _ptr(a)))

    def read_out_csr(self, weights=True):
        nr, ne = C.c_uint32(), C.c_uint64()
        _check(LIB.dtb_read_out_csr(self._h, C.byref(nr), C.byref(ne), None, None, None, None, None))
        nr, ne = nr.value, ne.value
        rows = np.empty(nr, np.uint32)
        ptr = np.empty(nr + 1, np.uint64)
        post = np.empty(ne, np.uint32)
        kind = np.empty(ne, np.uint8)
        w = np.empty((ne, 2), np.float32) if weights else None
        _check(LIB.dtb_read_out_csr(self._h, C.byref(C.c_uint32()), C.byref(C.c_uint64()), _ptr(rows), _ptr(ptr),
                                    _ptr(post), _ptr(kind), _ptr(w)))
        return rows, ptr, post, kind, w

    def save_state(self):
        size = C.c_uint64()
        _check(LIB.dtb_state_size(self._h, C.byref(size)))
        blob = np.empty(size.value, np.uint8)
        _check(LIB.dtb_save_state(self._h, _ptr(blob), size.value))
        return blob

    def load_state(self, blob):
        blob = np.ascontiguousarray(blob, np.uint8)
        _check(LIB.dtb_load_state(self._h, _ptr(blob), blob.shape[0]))


def _structured_c(spec, pop_id_base=0):
    """The C spec of a network.StructuredSpec plus the arrays it points into (keep them alive)."""
    keep = (_u32(spec.pop_sizes), _u32(spec.pop_exc), np.ascontiguousarray(spec.src_cdf, np.uint64),
            np.ascontiguousarray(spec.property_rows(), np.float32))
    s = StructuredSpecC(spec.n_pops, keep[0].ctypes.data, keep[1].ctypes.data, keep[2].ctypes.data,
                        keep[3].ctypes.data, pop_id_base, spec.in_degree, spec.seed, int(spec.dyadic_weights))
    return s, keep


class Server:
    """A pool of networks under an HBM cap serving a trace of simulate-window requests
    (dtb_server_*): continuous batching or one request at a time."""

    def __init__(self, hbm_cap_bytes=None, slice_steps=100, max_batch=64, syn_mode=SYN_PUSH, use_ou=True,
                 autotune=True):
        o = ServerOptions()
        LIB.dtb_server_default_options(C.byref(o))
        if hbm_cap_bytes is not None:
            o.hbm_cap_bytes = int(hbm_cap_bytes)
        o.slice_steps, o.max_batch, o.syn_mode = slice_steps, max_batch, syn_mode
        o.flags = RUN_USE_OU if use_ou else 0
        o.autotune = int(autotune)
        h = C.c_void_p()
        _check(LIB.dtb_server_create(C.byref(o), C.byref(h)))
        self._h = h
        self.n_pops = []

    def add_structured(self, spec, **opts):
        s, keep = _structured_c(spec)
        o = default_options(**opts)
        nid = C.c_uint32()
        _check(LIB.dtb_server_add_structured(self._h, C.byref(s), C.byref(o), C.byref(nid)))
        self.n_pops.append(spec.n_pops)
        return nid.value

    def add_npz(self, path, n_pops, **opts):
        o = default_options(**opts)
        nid = C.c_uint32()
        _check(LIB.dtb_server_add_npz(self._h, os.fsencode(path), C.byref(o), C.byref(nid)))
        self.n_pops.append(n_pops)
        return nid.value

    def play(self, requests, policy=SERVE_BATCHED):
        """requests: dicts {net, iters, arrival_s, ou: (mean, sigma, tau) arrays or None}, sorted by
        arrival.  Returns dicts with freqs [iters, P], start_s, finish_s, latency_s, events."""
        arr = (Request * len(requests))()
        keep, freqs = [], []
        for i, r in enumerate(requests):
            P = self.n_pops[r["net"]] if 0 <= r["net"] < len(self.n_pops) else 1   # the library rejects unknown ids
            fr = np.zeros((r["iters"], P), np.int32)
            freqs.append(fr)
            arr[i].net, arr[i].iters, arr[i].arrival_s = r["net"], r["iters"], float(r["arrival_s"])
            arr[i].freqs = fr.ctypes.data
            if r.get("ou") is not None:
                m, sd, tau = (np.ascontiguousarray(x, np.float32) for x in r["ou"])
                keep.extend((m, sd, tau))
                arr[i].ou_mean, arr[i].ou_sigma, arr[i].ou_tau = m.ctypes.data, sd.ctypes.data, tau.ctypes.data
        _check(LIB.dtb_server_play(self._h, len(requests), arr, policy))
        return [dict(freqs=freqs[i], start_s=arr[i].start_s, finish_s=arr[i].finish_s,
                     latency_s=arr[i].finish_s - arr[i].arrival_s, events=int(arr[i].events), status=arr[i].status)
                for i in range(len(requests))]

    def info(self):
        inf = ServerInfo()
        _check(LIB.dtb_server_info(self._h, C.byref(inf)))
        return {f: getattr(inf, f) for f, _ in ServerInfo._fields_}

    # ---- online serving (dtb_server_start / submit / poll / stop)
    def start(self, policy=SERVE_BATCHED):
        self._pending = {}
        _check(LIB.dtb_server_start(self._h, policy))

    def submit(self, net, iters, ou=None):
        """Submit a request now (thread-safe); returns its ticket."""
        P = self.n_pops[net] if 0 <= net < len(self.n_pops) else 1
        req = Request()
        req.net, req.iters = net, iters
        fr = np.zeros((iters, P), np.int32)
        req.freqs = fr.ctypes.data
        keep = [fr]
        if ou is not None:
            m, sd, tau = (np.ascontiguousarray(x, np.float32) for x in ou)
            keep.extend((m, sd, tau))
            req.ou_mean, req.ou_sigma, req.ou_tau = m.ctypes.data, sd.ctypes.data, tau.ctypes.data
        t = C.c_uint64()
        _check(LIB.dtb_server_submit(self._h, C.byref(req), C.byref(t)))
        self._pending[t.value] = (req, fr, keep)
        return t.value

    def poll(self, ticket, wait_s=0.0):
        """None while the request runs; its result dict once done."""
        done = C.c_int32()
        _check(LIB.dtb_server_poll(self._h, ticket, int(wait_s * 1000), C.byref(done)))
        if not done.value:
            return None
        req, fr, _ = self._pending.pop(ticket)
        return dict(freqs=fr, start_s=req.start_s, finish_s=req.finish_s, arrival_s=req.arrival_s,
                    latency_s=req.finish_s - req.arrival_s, events=int(req.events), status=req.status)

    def wait(self, ticket, timeout_s=600.0):
        """Block until the request is done (or raise after timeout_s)."""
        import time
        end = time.monotonic() + timeout_s
        while True:
            r = self.poll(ticket, wait_s=min(1.0, max(0.0, end - time.monotonic())))
            if r is not None:
                return r
            if time.monotonic() >= end:
                raise TimeoutError(f"request {ticket} not done after {timeout_s} s")

    def stop(self):
        _check(LIB.dtb_server_stop(self._h))

    def close(self):
        if self._h is not None and self._h.value:
            _check(LIB.dtb_server_destroy(self._h))
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Batch:
    """Several engines advanced together (dtb_batch_*): one launch per kernel per step."""

    def __init__(self, engines, graph=True):
        self.engines = list(engines)
        arr = (C.c_void_p * len(self.engines))(*[e._h.value for e in self.engines])
        h = C.c_void_p()
        _check(LIB.dtb_batch_create(arr, len(self.engines), C.byref(h)))
        self._h = h
        self.set_graph(graph)

    def set_graph(self, enable):
        _check(LIB.dtb_batch_set_graph(self._h, int(enable)))

    def set_push_variant(self, kind, param=0):
        """As Engine.set_push_variant, for the batch's shared push launch."""
        _check(LIB.dtb_batch_set_push_variant(self._h, kind, param))

    def info(self):
        n, g, k, p = C.c_uint32(), C.c_uint32(), C.c_int32(), C.c_int32()
        _check(LIB.dtb_batch_info(self._h, C.byref(n), C.byref(g), C.byref(k), C.byref(p)))
        return dict(members=n.value, graph_launches=g.value, push_kind=k.value, push_param=p.value)

    def run(self, iters, use_ou=True, freq=True, vmean=False, record_spikes=False,
            prop_mode=PROP_THRESHOLD, syn_mode=SYN_PUSH, outs=None, sample_spike=False):
        flags = (RUN_USE_OU if use_ou else 0) | (RUN_FREQ if freq else 0) | \
                (RUN_VMEAN if vmean else 0) | (RUN_RECORD_SPIKES if record_spikes else 0) | \
                (RUN_SAMPLE_SPIKE if sample_spike else 0)
        rq = RunRequest(iters, flags, prop_mode, syn_mode)
        m = len(self.engines)
        res = (RunOutput * m)()
        keep = []
        for i, e in enumerate(self.engines):
            if outs is not None:
                fr, vm = outs[i]
            else:
                fr = np.zeros((iters, e.n_pops), np.int32) if freq else None
                vm = np.zeros((iters, e.n_pops), np.float32) if vmean else None
            sb = np.zeros((iters, (e.n + 31) // 32), np.uint32) if record_spikes else None
            ss = np.zeros((iters, getattr(e, "n_sample_list", 0)), np.uint8) if sample_spike else None
            keep.append((fr, vm, sb, ss))
            res[i].sample_spike = None if ss is None else ss.ctypes.data
            res[i].freqs = None if fr is None else fr.ctypes.data
            res[i].vmeans = None if vm is None else vm.ctypes.data
            res[i].spike_bits = None if sb is None else sb.ctypes.data
        _check(LIB.dtb_batch_run(self._h, C.byref(rq), res))
        out = []
        for i, (fr, vm, sb, ss) in enumerate(keep):
            spikes = None
            if sb is not None:
                n = self.engines[i].n
                spikes = np.unpackbits(sb.view(np.uint8), axis=1, bitorder="little")[:, :n].astype(bool)
            out.append(RunResult(fr, vm, spikes, int(res[i].events), float(res[i].device_ms),
                                 tuple(res[i].kernel_ms), int(res[i].launches), ss))
        return out

    def close(self):
        if self._h is not None and self._h.value:
            _check(LIB.dtb_batch_destroy(self._h))
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
