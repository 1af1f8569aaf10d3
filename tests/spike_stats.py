"""Firing-rate and inter-spike-interval statistics of spike rasters, for the
long statistical parity runs.  Shared by the CPU tests (checked against the C
oracle's running moments) and the GPU tests (fed the engine's recorded spikes).

Conventions (the same as ``oracle_run_events`` in oracle/dtb_oracle.c): steps are
0-based absolute indices; a spike counts from step ``warm`` on; an inter-spike
interval counts when both of its spikes are at steps >= ``warm``; the pooled ISI
CV is std / mean over every such interval of every neuron.
"""
from __future__ import annotations

import numpy as np


class IsiMoments:
    """Running pooled ISI moments over raster chunks fed in step order."""

    def __init__(self, n, warm):
        self.n = n
        self.warm = warm
        self.last = np.full(n, -1, np.int64)
        self.count = 0
        self.s1 = 0.0
        self.s2 = 0.0

    def add(self, raster, t0):
        """raster: bool [k, n] of steps t0 .. t0 + k - 1."""
        neuron, step = np.nonzero(np.ascontiguousarray(raster.T))   # neuron-major, steps ascending
        if neuron.size == 0:
            return
        step = step.astype(np.int64) + t0
        prev = np.empty_like(step)
        first = np.ones(neuron.size, bool)
        first[1:] = neuron[1:] != neuron[:-1]
        prev[~first] = step[np.nonzero(~first)[0] - 1]
        prev[first] = self.last[neuron[first]]
        ok = (prev >= self.warm) & (step >= self.warm)
        d = (step - prev)[ok].astype(np.float64)
        self.count += int(d.size)
        self.s1 += float(d.sum())
        self.s2 += float((d * d).sum())
        last = np.ones(neuron.size, bool)
        last[:-1] = neuron[1:] != neuron[:-1]
        self.last[neuron[last]] = step[last]

    def cv(self):
        if self.count < 2:
            return float("nan")
        mean = self.s1 / self.count
        return float(np.sqrt(max(self.s2 / self.count - mean * mean, 0.0)) / mean)


def population_rates(counts, sizes, dt_ms, warm):
    """Rates in Hz per population from per-step counts [steps, P] (steps >= warm)."""
    c = np.asarray(counts, np.int64)[warm:].sum(0)
    return c / np.asarray(sizes, np.float64) / ((np.asarray(counts).shape[0] - warm) * dt_ms * 1e-3)
