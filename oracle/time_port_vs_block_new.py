"""Time the C port of the reference model (oracle/dtb_oracle.c, the CPU baseline
that bench.py runs) against the reference's own ``models/block_new.py`` on the
same network, same threads, same step count -- the speed ratio that relates the
bench's CPU figures to the reference implementation itself.

block_new takes its weights as one ``torch.sparse_coo`` tensor [4, N, N] (the
receptor pair of every synapse as two nonzeros), the form it needs above a few
thousand neurons, and runs its ``run(debug_mode=False)`` loop as shipped,
including the per-population statistics loop (block_new.py:152-156).

Needs the reference checkout (this container only; nothing here travels):
    python oracle/time_port_vs_block_new.py /path/to/Digital_twin_brain-open [steps]
"""
import importlib.util
import os
import sys
import time

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)

import __graft_entry__  # noqa: E402

__graft_entry__.load_package()
from dtb_b200 import network as nw  # noqa: E402
from oracle import c_oracle as cc  # noqa: E402
from oracle import lif_oracle as lo  # noqa: E402

# the bench's CPU sample: 50,000 neurons, 20 populations, in-degree 1000 (bench.py CPU_SAMPLE)
N, POPS, DEGREE, SEED, BURN = 50_000, 20, 1000, 7, 600


def load_block_new(ref_root):
    spec = importlib.util.spec_from_file_location("block_new_ref", os.path.join(ref_root, "models", "block_new.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def sparse_w(net, n):
    ch = np.where(net["input_channel_offset"] != 0, 2, 0).astype(np.int64)
    post = net["output_neuron_idx"].astype(np.int64)
    pre = net["input_neuron_idx"].astype(np.int64)
    idx = np.stack([np.concatenate([ch, ch + 1]), np.concatenate([post, post]), np.concatenate([pre, pre])])
    val = np.concatenate([net["weight"][:, 0], net["weight"][:, 1]])
    return torch.sparse_coo_tensor(torch.from_numpy(idx), torch.from_numpy(val), (4, n, n)).coalesce()


def main(ref_root, steps):
    threads = os.cpu_count()
    torch.set_num_threads(threads)
    block_new = load_block_new(ref_root)
    spec = nw.structured_spec(N, POPS, DEGREE, SEED)
    net = cc.structured_edges(spec)
    z, _ = lo.torch_noise_stream(0, N, BURN + steps, False)

    # the port carries the network past its quiet start; block_new then continues from the
    # port's state on the same noise stream (its global generator advanced past the burn-in draws)
    port = cc.COracle(net)
    port.run(z[:BURN], record=False)
    state = dict(V=port.V.copy(), J=port.J.copy(), t_last=port.t_last.copy(), i_bg=port.i_bg.copy(),
                 I_syn=port.I_syn.copy(), t=float(port.t[0]))
    t0 = time.perf_counter()
    sp_port, _, ev_port = port.run(z[BURN:], record=True)
    port_s = time.perf_counter() - t0

    w = sparse_w(net, N)
    b = block_new.block(torch.from_numpy(net["property"]), w, delta_t=0.1, i_mean=0.6, i_sigma=0.2, tau_i=10.0)
    b.V_i = torch.from_numpy(state["V"])
    b.J_ui = torch.from_numpy(state["J"])
    b.t_ik_last = torch.from_numpy(state["t_last"])
    b.i_background = torch.from_numpy(state["i_bg"])
    b.I_syn = torch.from_numpy(state["I_syn"])
    b.t = torch.tensor(state["t"], dtype=torch.float32)
    torch.manual_seed(0)
    for _ in range(BURN):
        torch.randn(N)
    out_deg = np.bincount(net["input_neuron_idx"], minlength=N)
    ref_sp, ev_ref = [], 0
    t0 = time.perf_counter()
    for _ in range(steps):
        b.run(False)
        a = b.active.numpy().copy()
        ref_sp.append(a)
        ev_ref += int(out_deg[a].sum())
    ref_s = time.perf_counter() - t0
    agree = float((np.array(ref_sp) == sp_port).mean())
    print(f"network: {N} neurons, {POPS} populations, in-degree {DEGREE} ({N * DEGREE:.2e} synapses), "
          f"{threads} threads, torch {torch.__version__}; {steps} steps after a {BURN}-step burn-in")
    print(f"block_new (sparse COO, as shipped): {1e3 * ref_s / steps:.1f} ms/step, {ev_ref / ref_s:.3e} events/s "
          f"({sum(int(x.sum()) for x in ref_sp)} spikes)")
    print(f"C port:                             {1e3 * port_s / steps:.1f} ms/step, {ev_port / port_s:.3e} events/s "
          f"({int(sp_port.sum())} spikes)")
    print(f"port / block_new speed:             {ref_s / port_s:.0f}x; spike rasters agree on {100 * agree:.4f} % "
          f"of neuron-steps")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("DTB_REFERENCE", ""),
         int(sys.argv[2]) if len(sys.argv) > 2 else 10)
