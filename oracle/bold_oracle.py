"""CPU restatement of the reference's Balloon-Windkessel BOLD model -- TEST
INFRASTRUCTURE ONLY (tests/ use it as the checker of the CUDA kernel).

Follows models/bold_model_pytorch.py:61-96 (``BOLD.run``) in float32 with the
same operation order: each state variable is advanced in place, in the order
q, v, f_in, s, so q's update reads the old v and f_in, f_in's reads the old s,
and the output reads the new q and v; the Python-float parameters enter as
float32 scalars; divisions by parameters are true divisions; ``x ** y`` is a
float32 power.  Initial state (``run`` with no state set): s = 0, q = 0,
v = 1, f_in = 1.  Pinned by tests/golden/bold_*.npz (made by running the
reference module, tests/golden/make_bold_golden.py).
"""
import numpy as np

F = np.float32


class BoldOracle:
    def __init__(self, epsilon, tao_s, tao_f, tao_0, alpha, E_0, V_0, delta_t=1e-3, n=None, state=None):
        self.epsilon, self.tao_s, self.tao_f, self.tao_0 = F(epsilon), F(tao_s), F(tao_f), F(tao_0)
        self.E_0, self.V_0, self.dt = F(E_0), F(V_0), F(delta_t)
        div_alpha = 1 / alpha                       # Python float, as in BOLD.__init__
        self.div_alpha = F(div_alpha)
        self.div_alpha_m1 = F(div_alpha - 1)
        self.one_m_e0 = F(1 - E_0)                  # (1 - self.E_0) is a Python float
        self.e0_term = F(2 * E_0 - 0.2)             # (2 * self.E_0 - 0.2)
        self.seven_e0 = F(7 * E_0)                  # 7 * self.E_0
        if state is not None:
            self.s, self.q, self.v, self.f_in = (np.array(x, F) for x in state)
        else:
            self.s = np.zeros(n, F)
            self.q = np.zeros(n, F)
            self.v = np.ones(n, F)
            self.f_in = np.ones(n, F)

    def run(self, u):
        u = np.asarray(u, F)
        with np.errstate(divide="ignore", over="ignore", invalid="ignore"):
            d_s = (self.epsilon * u - self.s / self.tao_s) - (self.f_in - F(1)) / self.tao_f
            q_part = np.where(self.f_in > 0, F(1) - np.power(self.one_m_e0, F(1) / self.f_in), F(1)).astype(F)
            dq = (self.f_in * q_part / self.E_0 - self.q * np.power(self.v, self.div_alpha_m1)) / self.tao_0
            self.q = (self.q + dq * self.dt).astype(F)
            dv = (self.f_in - np.power(self.v, self.div_alpha)) / self.tao_0
            self.v = (self.v + dv * self.dt).astype(F)
            self.f_in = (self.f_in + self.s * self.dt).astype(F)
            self.f_in = np.where(self.f_in > 0, self.f_in, F(0)).astype(F)
            self.s = (self.s + d_s * self.dt).astype(F)
            out = self.V_0 * ((self.seven_e0 * (F(1) - self.q) + F(2) * (F(1) - self.q / self.v))
                              + self.e0_term * (F(1) - self.v))
        return out.astype(F)

    def state(self):
        return np.stack([self.s, self.q, self.v, self.f_in])


# DA_voxel.py:470-476
DA_PARAMS = dict(epsilon=200, tao_s=0.8, tao_f=0.4, tao_0=1, alpha=0.2, E_0=0.8, V_0=0.02)


def bold_inputs(n, steps, seed):
    """Seeded voxel activity for the BOLD fixtures: a slow random walk around 0.1
    (spikes per neuron per step at a few hundred Hz), floored at 1e-5 as DA_voxel.py:330 does."""
    rng = np.random.default_rng(seed)
    walk = np.cumsum(rng.standard_normal((steps, n)), axis=0) / 20.0
    return np.maximum(0.1 + 0.05 * walk, 1e-5).astype(np.float32)


def da_filter(w_hat, bold_y, noise, hp_num, bold_sigma, rate=0.5):
    """Ensemble Kalman update of DA_voxel.filter (data_assimilation/DA_voxel.py:289-307),
    float32 in, reductions and products accumulated in float64, result rounded once.

    w_hat [E, V, S] (S = hp_num + 6, the BOLD signal last), bold_y [V] the observation,
    noise [E, V] the standard-normal draws the reference takes from torch.normal (scaled
    by sqrt(bold_sigma) here as there).  Returns w [E, V, S] float32.
    """
    w_hat = np.asarray(w_hat, np.float64)
    E, V, S = w_hat.shape
    assert S == hp_num + 6
    w_mean = w_hat.mean(axis=0, keepdims=True)
    w_diff = w_hat - w_mean
    w_cxx = (w_diff[:, :, -1] ** 2).sum(axis=0) / (E - 1) + bold_sigma
    temp = w_diff[:, :, -1] / w_cxx[None, :] / (E - 1)
    innov = np.asarray(bold_y, np.float64)[None, :] + np.sqrt(bold_sigma) * np.asarray(noise, np.float64) - w_hat[:, :, -1]
    w = w_hat + rate * innov[:, :, None] * (temp[:, :, None] * w_diff).sum(axis=0, keepdims=True)
    g = (innov @ temp.T) / V
    w = w + (1 - rate) * (g @ w_diff.reshape(E, V * S)).reshape(E, V, S)
    return w.astype(np.float32)
