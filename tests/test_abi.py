"""The C-ABI library: loads without a GPU, exports every declared symbol, host-only
entry points behave, and device entry points fail cleanly when no device exists."""
import os
import re

import numpy as np
import pytest

from conftest import ROOT, has_gpu
from dtb_b200 import engine as E
from dtb_b200 import network as nw
from oracle import csr_oracle as co

HEADER = os.path.join(ROOT, "include", "dtb_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dtb_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(E.LIB, name), f"{name} declared in dtb_b200.h but not exported"


def test_binding_covers_the_header():
    assert set(declared_functions()) == set(E.SIGNATURES)


def test_versions_and_status_strings():
    assert E.LIB.dtb_abi_version() == 2
    v = E.LIB.dtb_engine_version()
    assert (v // 1000, (v % 1000) // 100, v % 100) == (1, 0, 0)
    assert E.status_string(0) == "SNN_OK"
    assert E.status_string(5) == "SNN_INVALID_NETWORK"
    assert E.status_string(16) == "DTB_OUT_OF_MEMORY"


def test_default_options():
    o = E.default_options()
    assert abs(o.dt - 0.1) < 1e-7 and o.build_push == 1 and o.build_pull == 0
    assert abs(o.ou_mean - 0.6) < 1e-7 and abs(o.ou_tau - 10.0) < 1e-6


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_create_without_device_reports_no_device():
    with pytest.raises(E.DtbError) as ei:
        E.Engine.from_arrays(nw.make_uniform_block(64, 4))
    assert ei.value.status == E.NO_DEVICE


def test_invalid_arguments_are_statuses_not_crashes():
    import ctypes as C
    h = C.c_void_p()
    assert E.LIB.dtb_create(None, None, C.byref(h)) == E.INVALID_PARAMETER
    assert E.LIB.dtb_destroy(None) == E.INVALID_PARAMETER
    assert E.LIB.dtb_run(None, None, None) == E.INVALID_PARAMETER
    o = E.default_options()
    assert E.LIB.dtb_create_from_npz(b"", C.byref(o), C.byref(h)) == E.INVALID_PARAMETER


@pytest.mark.skipif(has_gpu(), reason="argument check only; no device calls")
def test_compaction_rejects_counts_beyond_32_bits():
    """Bitmaps whose tile or word counts would wrap 32 bits are rejected before any
    CUDA call (the pointers are never touched, so placeholders suffice here)."""
    import ctypes as C
    fake = C.c_void_p(256)
    for n in (0xFFFFFFFF, 0xFFFFF001):
        assert E.LIB.dtb_compact_spikes(fake, n, fake, fake, None) == E.INVALID_PARAMETER
        assert "limit" in E.LIB.dtb_last_error().decode()
    assert E.LIB.dtb_compact_spikes_noalloc(fake, (1 << 26) + 1, fake, fake, None) == E.INVALID_PARAMETER


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_host_csr_matches_oracle(seed):
    """The engine's host CSR builder equals the restated reference builder, bit for bit."""
    net = nw.make_uniform_block(700, 15, seed=seed)
    rng = np.random.default_rng(seed)
    perm = rng.permutation(net["input_neuron_idx"].shape[0])   # any input order
    shuffled = {k: (v[perm] if k != "property" else v) for k, v in net.items()}
    ref = co.reference_out_csr(shuffled)
    rows, ptr, post, kind, p = E.build_out_csr_host(700, shuffled["input_neuron_idx"],
                                                    shuffled["output_neuron_idx"],
                                                    shuffled["input_channel_offset"])
    assert np.array_equal(rows, ref["rows"])
    assert np.array_equal(ptr, ref["row_ptr"])
    assert np.array_equal(post, ref["post"])
    assert np.array_equal(kind, ref["kind"])
    assert np.array_equal(p, ref["perm"])


def test_host_csr_edge_cases():
    # empty network, isolated neurons, a single hub row
    rows, ptr, post, kind, p = E.build_out_csr_host(10, np.zeros(0), np.zeros(0), np.zeros(0))
    assert rows.size == 0 and list(ptr) == [0] and post.size == 0
    pre = np.array([7, 7, 7, 7])
    post_in = np.array([1, 0, 3, 1])
    rows, ptr, post, kind, p = E.build_out_csr_host(10, pre, post_in, np.array([0, 2, 0, 2]))
    assert list(rows) == [7] and list(ptr) == [0, 4] and list(post) == [1, 0, 3, 1] and list(kind) == [0, 1, 0, 1]
    with pytest.raises(E.DtbError):
        E.build_out_csr_host(5, np.array([5]), np.array([0]), np.array([0]))


def test_server_rejects_bad_traces_without_a_device():
    """Trace validation happens before any device work."""
    with E.Server() as srv:
        with pytest.raises(E.DtbError) as ei:
            srv.play([dict(net=0, iters=10, arrival_s=0.0)])     # no such network
        assert ei.value.status == E.INVALID_PARAMETER
        srv.n_pops.append(3)                                       # pretend a network of 3 populations
        with pytest.raises(E.DtbError):
            srv.play([dict(net=0, iters=10, arrival_s=0.0)])     # still unknown to the library
    import ctypes as C
    o = E.ServerOptions()
    E.LIB.dtb_server_default_options(C.byref(o))
    assert o.slice_steps == 100 and o.max_batch == 64 and o.hbm_cap_bytes == 150 * 10**9
    o.slice_steps = 0
    h = C.c_void_p()
    assert E.LIB.dtb_server_create(C.byref(o), C.byref(h)) == E.INVALID_PARAMETER


def test_npz_directory_must_agree_with_the_weight_dtype(tmp_path):
    """The weight type named by the path's directory (src/configuration.cpp:1411-1435)
    must match the file's dtype; the check happens before any device work."""
    net = nw.make_uniform_block(50, 5, seed=1)
    d = tmp_path / "half"
    os.makedirs(d)
    nw.write_npz(str(d / "block_0.npz"), net)             # float32 weights under half/
    with pytest.raises(E.DtbError) as ei:
        E.Engine.from_npz(str(d / "block_0.npz"))
    assert ei.value.status == E.INVALID_NETWORK and "/half" in str(ei.value)
