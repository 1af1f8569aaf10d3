"""CPU oracle for the DTB per-timestep hot path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
may import this module, and only as the checker.  The product path (the CUDA
engine behind ``include/dtb_b200.h``) never calls it.

This is a numpy restatement of the reference CPU model ``models/block_new.py``:

* ``block.run``              (block_new.py:122-158)  ->  ``LifOracle.step``
* ``update_i_background``    (block_new.py:92-96)    OU current, one N(0,1) draw per neuron
* ``update_Vi``              (block_new.py:104-117)  Euler step, refractory clamp, threshold
* ``update_J_ui`` / ``bmm``  (block_new.py:71-84)    J = J*exp(-dt/tau) + W.s
* ``update_I_syn``           (block_new.py:86-90)    I = sum_u g_u (V_u - V) J_u
* ``update_t_ik_last``       (block_new.py:119-120)
* per-population outputs     (block_new.py:152-158)

Float32 arithmetic follows block_new's torch op order exactly: ``-dt/tau`` is
evaluated as ``reciprocal(tau) * -dt`` (torch's ``__rtruediv__``), the receptor
sum is sequential ``((I0+I1)+I2)+I3`` (torch's dim-0 reduction), ``t`` is a
float32 scalar advanced by ``t += dt`` each step.  The per-population constants
``exp(.)`` and ``sqrt(.)`` are evaluated in float64 and rounded once to float32
(for the parameters used here that equals torch's result; see
tests/test_oracle.py).  ``W.s`` is accumulated in float64 per post neuron in
in-edge order and rounded once; with dyadic weights (multiples of 1/256) every
order gives the same float32 sum, which is what the bit-exact tests use.

Noise: block_new draws ``torch.randn(N)`` each step and, in debug mode, then
``torch.rand(N)``, from torch's global CPU generator.  ``torch_noise_stream``
replays that call sequence so the oracle (and the GPU engine, through its
injected-noise mode) sees the reference's exact draws.

Propagation modes:
* ``PROP_THRESHOLD`` -- block_new ``run(debug_mode=False)``: threshold spikes drive J;
* ``PROP_NOISE``     -- block_new ``run(debug_mode=True, noise_rate)``: the noise
  train ``u < noise_rate`` replaces the propagated spikes (block_new.py:143-146);
* ``PROP_OR``        -- the reference C++ engine with OU off: the noise train is
  OR-ed into the threshold spikes (``src/stage/spike.cpp:42-68``).
In every mode the threshold spikes set t_last and the population counts.

``dtype=np.float64`` gives the FP64 oracle (every constant, state and weight in
float64, dt = 0.1 in double), used to state the error of the FP32 and BF16 forms.
"""
from __future__ import annotations

import numpy as np

PROP_THRESHOLD = 0
PROP_NOISE = 1
PROP_OR = 2


def _f(dtype, x):
    return np.asarray(x, dtype=dtype)


def decay_constants(tau, dt, dtype=np.float32):
    """exp(-dt/tau) as block_new evaluates it: reciprocal(tau) * (-dt), then exp."""
    tau = _f(dtype, tau)
    x = (_f(dtype, 1.0) / tau) * _f(dtype, -dt)
    return _f(dtype, np.exp(x.astype(np.float64)))


def ou_constants(tau, sigma, dt, dtype=np.float32):
    """(1 - exp(-dt/tau), sqrt(1 - exp(-2 dt/tau)) * sigma), block_new.py:93-95."""
    tau = _f(dtype, tau)
    r = _f(dtype, 1.0) / tau
    e1 = _f(dtype, np.exp((r * _f(dtype, -dt)).astype(np.float64)))
    e2 = _f(dtype, np.exp((r * _f(dtype, -2.0 * dt)).astype(np.float64)))
    f1 = _f(dtype, 1.0) - e1
    f2 = _f(dtype, np.sqrt((_f(dtype, 1.0) - e2).astype(np.float64)))
    return f1, f2 * _f(dtype, sigma)


def torch_noise_stream(seed, n, steps, with_uniform):
    """Replay block_new's RNG calls: per step randn(N), then rand(N) in debug mode.

    Returns (z [steps, n] float32, u [steps, n] float32 or None).
    """
    import torch
    g = torch.Generator()
    g.manual_seed(seed)
    z = np.empty((steps, n), np.float32)
    u = np.empty((steps, n), np.float32) if with_uniform else None
    for s in range(steps):
        z[s] = torch.randn(n, generator=g).numpy()
        if with_uniform:
            u[s] = torch.rand(n, generator=g).numpy()
    return z, u


def torch_noise_chunks(seed, n, steps, chunk, with_uniform=False):
    """The stream of ``torch_noise_stream`` in chunks of at most ``chunk`` steps
    (same call order, so the concatenated chunks equal its arrays), for runs too
    long to hold every draw at once.  Yields (z, u or None)."""
    import torch
    g = torch.Generator()
    g.manual_seed(seed)
    done = 0
    while done < steps:
        k = min(chunk, steps - done)
        z = np.empty((k, n), np.float32)
        u = np.empty((k, n), np.float32) if with_uniform else None
        for s in range(k):
            z[s] = torch.randn(n, generator=g).numpy()
            if with_uniform:
                u[s] = torch.rand(n, generator=g).numpy()
        done += k
        yield z, u


class LifOracle:
    """One LIF block, stepping exactly like block_new (see module docstring).

    ``net`` is a dict in the reference's npz key set.  ``ou`` maps to per-neuron
    (mean, sigma, tau) arrays or scalars.  ``prop_mode`` selects what drives J.
    """

    def __init__(self, net, dt=0.1, ou=(0.6, 0.2, 10.0), dtype=np.float32,
                 prop_mode=PROP_THRESHOLD):
        self.dtype = dt_ = dtype
        prop = np.asarray(net["property"])
        n = prop.shape[0]
        self.n = n
        self.dt = dt
        self.prop_mode = prop_mode
        P = prop.astype(dt_)
        self.noise_rate = P[:, 0]
        self.blocked = prop[:, 1] != 0
        self.i_ext = P[:, 2]
        self.pop = prop[:, 3].astype(np.int64)
        C, T_ref, g_L, V_L, V_th, V_reset = (P[:, c] for c in range(4, 10))
        self.g_u = P[:, 10:14].T.copy()          # [4, N]
        self.V_u = P[:, 14:18].T.copy()          # [4, N]
        tau_u = P[:, 18:22].T.copy()
        self.decay = decay_constants(tau_u, dt, dt_)
        self.dtC = (_f(dt_, 1.0) / C) * _f(dt_, dt)
        self.neg_gL = -g_L
        self.V_L, self.V_th, self.V_reset, self.T_ref = V_L, V_th, V_reset, T_ref
        mean, sigma, tau_i = (np.broadcast_to(_f(dt_, x), (n,)).copy() for x in ou)
        self.ou_mean = mean
        self.ou_f1, self.ou_f2s = ou_constants(tau_i, sigma, dt, dt_)
        # state (block_new.py:41, 57-62)
        self.i_bg = mean.copy()
        self.t_last = -T_ref.copy()
        self.V = (V_th + V_reset) / _f(dt_, 2.0)
        self.J = np.zeros((4, n), dt_)
        self.t = _f(dt_, 0.0)
        self.I_syn = np.zeros(n, dt_)
        self.I_u = np.zeros((4, n), dt_)
        # in-edges, post-major (the file order)
        pre = np.asarray(net["input_neuron_idx"], np.int64)
        post = np.asarray(net["output_neuron_idx"], np.int64)
        ch = np.where(np.asarray(net["input_channel_offset"]) != 0, 2, 0).astype(np.int64)
        w = np.asarray(net["weight"]).astype(np.float64)
        self._pre = pre
        self._slot0 = ch * n + post
        self._slot1 = (ch + 1) * n + post
        self._w0 = w[:, 0]
        self._w1 = w[:, 1]
        self.steps_done = 0

    def set_property(self, prop):
        """Re-read the neuron parameters from a new property matrix (state kept),
        as ``block.update_property`` does (block_new.py:160-178)."""
        d = self.dtype
        P = np.asarray(prop).astype(d)
        self.noise_rate = P[:, 0]
        self.i_ext = P[:, 2]
        C, T_ref, g_L, V_L, V_th, V_reset = (P[:, c] for c in range(4, 10))
        self.g_u = P[:, 10:14].T.copy()
        self.V_u = P[:, 14:18].T.copy()
        self.decay = decay_constants(P[:, 18:22].T.copy(), self.dt, d)
        self.dtC = (_f(d, 1.0) / C) * _f(d, self.dt)
        self.neg_gL = -g_L
        self.V_L, self.V_th, self.V_reset, self.T_ref = V_L, V_th, V_reset, T_ref

    def set_ou(self, mean, sigma, tau, mask=None):
        """Set the OU parameters of the neurons in ``mask`` (all by default)."""
        d = self.dtype
        m = np.ones(self.n, bool) if mask is None else mask
        self.ou_mean[m] = _f(d, mean)
        f1, f2s = ou_constants(np.full(int(m.sum()), tau, d), np.full(int(m.sum()), sigma, d), self.dt, d)
        self.ou_f1[m] = f1
        self.ou_f2s[m] = f2s

    def synaptic_input(self, s):
        """W.s: per-receptor input of the spikes ``s`` [N] bool, shape [4, N]."""
        m = s[self._pre]
        acc = np.bincount(self._slot0[m], weights=self._w0[m], minlength=4 * self.n)
        acc += np.bincount(self._slot1[m], weights=self._w1[m], minlength=4 * self.n)
        return acc.reshape(4, self.n).astype(self.dtype)

    def step(self, z, u=None):
        """Advance one step with normal draws ``z`` (and uniforms ``u`` for noise).

        Returns (active [N] bool, propagated [N] bool).
        """
        d = self.dtype
        z = np.asarray(z, d)
        self.t = _f(d, self.t + _f(d, self.dt))
        # update_i_background
        self.i_bg = self.i_bg + (self.ou_f1 * (self.ou_mean - self.i_bg) + self.ou_f2s * z)
        # update_Vi
        main = self.neg_gL * (self.V - self.V_L)
        cd = ((main + self.I_syn) + self.i_ext) + self.i_bg
        v_normal = self.V + self.dtC * cd
        not_sat = self.t >= (self.t_last + self.T_ref)
        v = np.where(not_sat, v_normal, self.V_reset)
        active = v >= self.V_th
        self.V = np.minimum(v, self.V_th)
        if self.prop_mode == PROP_THRESHOLD:
            prop = active
        else:
            noise = np.asarray(u, d) < self.noise_rate
            prop = noise if self.prop_mode == PROP_NOISE else (noise | active)
        # update_J_ui
        self.J = self.J * self.decay + self.synaptic_input(prop)
        # update_I_syn
        self.I_u = (self.g_u * (self.V_u - self.V)) * self.J
        self.I_syn = ((self.I_u[0] + self.I_u[1]) + self.I_u[2]) + self.I_u[3]
        # update_t_ik_last
        self.t_last = np.where(active, self.t, self.t_last)
        self.steps_done += 1
        return active, prop

    def step_substeps(self, zs):
        """One step of ``len(zs)`` substeps, the C++ engine's ``t_steps`` loop
        (tools/dist_simulator.cpp:2085-2112), on an oracle built with ``dt = dt_step /
        t_steps`` in float32 (src/block.cpp:304, 317, 668, 1275 derive every factor from
        ``delta_t_ / t_steps_``).  Each substep: OU, membrane update and threshold with
        block_new's equations, its spikes OR-ed into the step's record
        (``update_F_accumulated_spike_gpu``, src/block.cpp:729-737) and t_last set;
        between substeps J decays with no input and I_syn is recomputed
        (``update_J_presynaptic_per_step_gpu``, src/block.cpp:875-888); after the last,
        the recorded spikes are propagated once: J = J*decay + W.s.  Threshold
        propagation only (the reference requires the OU background for substeps,
        dist_simulator.cpp:3225-3234).  Returns the recorded spikes [N] bool.
        """
        d = self.dtype
        rec = np.zeros(self.n, bool)
        for k, z in enumerate(zs):
            self.t = _f(d, self.t + _f(d, self.dt))
            self.i_bg = self.i_bg + (self.ou_f1 * (self.ou_mean - self.i_bg) + self.ou_f2s * np.asarray(z, d))
            main = self.neg_gL * (self.V - self.V_L)
            cd = ((main + self.I_syn) + self.i_ext) + self.i_bg
            v_normal = self.V + self.dtC * cd
            v = np.where(self.t >= (self.t_last + self.T_ref), v_normal, self.V_reset)
            active = v >= self.V_th
            self.V = np.minimum(v, self.V_th)
            rec |= active
            self.t_last = np.where(active, self.t, self.t_last)
            if k + 1 < len(zs):
                self.J = self.J * self.decay
            else:
                self.J = self.J * self.decay + self.synaptic_input(rec)
            self.I_u = (self.g_u * (self.V_u - self.V)) * self.J
            self.I_syn = ((self.I_u[0] + self.I_u[1]) + self.I_u[2]) + self.I_u[3]
        self.steps_done += 1
        return rec

    def population_stats(self, active, pop_ids=None):
        """(spike count [P] int64, mean V [P] float64) over each population.

        Neurons flagged ``blocked_in_stat`` are excluded, as the reference's stat
        kernels do (src/stage/stat_result.cpp:161-299).
        """
        if pop_ids is None:
            pop_ids = np.unique(self.pop)
        keep = ~self.blocked
        counts = np.zeros(len(pop_ids), np.int64)
        vmean = np.zeros(len(pop_ids), np.float64)
        for k, p in enumerate(pop_ids):
            m = (self.pop == p) & keep
            counts[k] = int(active[m].sum())
            vmean[k] = float(self.V[m].astype(np.float64).mean()) if m.any() else 0.0
        return counts, vmean
