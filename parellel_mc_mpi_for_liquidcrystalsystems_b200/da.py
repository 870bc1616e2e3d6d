"""Learned volume-move screen and the P2 effective-sample-size measurement.

* :class:`Surrogate` - the 4097 -> 128 -> 128 -> 1 MLP of liblcmc.so (BF16
  tensor-core kernels), trained on (features, exact slope dU / (N delta))
  samples that plain NPT runs record;
* :func:`collect_samples` - run plain NPT replicas and record samples;
* :func:`p2_series` / :func:`ess` - the per-sweep P2 series of a replica and its
  effective sample size (integrated autocorrelation time with Sokal's automatic
  window, A. D. Sokal, "Monte Carlo methods in statistical mechanics", 1996).

No counterpart in the reference: MCnptColloid.c has no volume move
(system_pressure is parsed at MCnptColloid.c:3978 and never used).
"""
import ctypes as C

import numpy as np

from ._lib import FP, N_FEATURES, check, lib


class Surrogate:
    """The surrogate network; predicts the slope dU / (N delta) of a volume
    move, divided by `scale`, from the 4097 features of an end point."""

    def __init__(self, max_batch=512, seed=1):
        h = C.c_void_p()
        check(lib().lcmc_mlp_create(N_FEATURES, 128, max_batch, seed, C.byref(h)))
        self._h = h
        self.scale = 1.0
        self.history = []

    def close(self):
        if self._h:
            lib().lcmc_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def fit(self, x, slope, epochs=10, batch=256, lr=1e-3, seed=1, max_abs=1000.0):
        """Train on features x (n x 4097) and exact slopes dU / (N delta);
        targets are divided by their standard deviation (kept as `scale`).
        Samples with |slope| > max_abs (moves into overlaps, which stage 2
        rejects anyway) are left out: their R^12 energies would swamp the
        squared loss."""
        y = np.asarray(slope, dtype=np.float64)
        keep = np.isfinite(y) & (np.abs(y) <= max_abs)
        x = np.ascontiguousarray(np.asarray(x)[keep], dtype=np.float32)
        y = y[keep]
        if len(y) == 0:
            raise ValueError("no training sample with |slope| <= max_abs")
        self.scale = float(np.std(y)) or 1.0
        t = np.ascontiguousarray(y / self.scale, dtype=np.float32)
        loss = C.c_float()
        check(lib().lcmc_mlp_train(self._h, x.ctypes.data_as(FP), t.ctypes.data_as(FP), len(t), epochs, batch, lr,
                                   seed, C.byref(loss)))
        self.history.append(loss.value)
        return loss.value

    def predict(self, x):
        """Slope dU / (N delta) predicted for each feature row."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        out = np.zeros(len(x), dtype=np.float32)
        check(lib().lcmc_mlp_predict(self._h, x.ctypes.data_as(FP), len(x), out.ctypes.data_as(FP)))
        return out.astype(np.float64) * self.scale


def collect_samples(system, n_sweeps, capacity=None):
    """Run `n_sweeps` sweeps of a GBSystem (NPT replicas, plain volume moves)
    recording (features, exact dU / (N delta)) of every evaluated volume move."""
    system.record_volume_samples(capacity or n_sweeps * system.n_replicas)
    system.sweep(n_sweeps)
    x, y = system.get_volume_samples()
    system.record_volume_samples(0)
    return x, y


def p2_series(system, replica=0):
    """(sweep, P2, E, V) arrays from the recorded history of a replica."""
    rows = system.get_history(replica)
    N = system.params[replica].num_particles
    s = rows[:, 1:7] / N
    Q = np.empty((len(rows), 3, 3))
    Q[:, 0, 0], Q[:, 0, 1], Q[:, 0, 2] = s[:, 0] - 1 / 3, s[:, 1], s[:, 2]
    Q[:, 1, 1], Q[:, 1, 2], Q[:, 2, 2] = s[:, 3] - 1 / 3, s[:, 4], s[:, 5] - 1 / 3
    Q[:, 1, 0], Q[:, 2, 0], Q[:, 2, 1] = Q[:, 0, 1], Q[:, 0, 2], Q[:, 1, 2]
    p2 = 1.5 * np.linalg.eigvalsh(Q)[:, -1]
    return rows[:, 0], p2, rows[:, 7], rows[:, 8]


def integrated_autocorrelation_time(x, c=5.0):
    """tau_int = 1/2 + sum_t rho(t), summed up to the first window W >= c tau_int(W)
    (Sokal's automatic windowing); autocorrelation by FFT."""
    x = np.asarray(x, dtype=np.float64)
    n = len(x)
    if n < 4:
        return 0.5
    y = x - x.mean()
    var = np.dot(y, y) / n
    if var == 0:
        return 0.5
    f = np.fft.rfft(y, 2 * n)
    acf = np.fft.irfft(f * np.conj(f))[:n] / (n * var)
    tau = 0.5
    for w in range(1, n):
        tau += acf[w]
        if w >= c * tau:
            return max(tau, 0.5)
    return max(tau, 0.5)


def ess(x, c=5.0):
    """Effective sample size n / (2 tau_int)."""
    return len(x) / (2.0 * integrated_autocorrelation_time(x, c))
