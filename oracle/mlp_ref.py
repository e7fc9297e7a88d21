"""CPU oracle of the learned settling-velocity network (test infrastructure).

Only the tests, the smoke entry and the benchmark's CPU baseline use this
module; the product path never does.  It restates in numpy FP64:

  * the network 5 -> 64 -> 64 -> 1 with tanh, parameters laid out as the
    library's vector (W1[64][5], b1, W2[64][64], b2, W3[64], b3);
  * the mean-squared-error loss and its gradient by hand-written
    back-propagation (the check of the device training kernel);
  * the feature map and output transform of the surrogate, from the
    normalisation constants the library reports;
  * the counter-based draw of the training samples (SplitMix64 finaliser,
    Steele, Lea & Flood 2014), so the device's samples can be re-labelled
    here by the drag-law iteration of phys_get_vset_point
    (mod_Phys.F90:757-954, restated in f3d_oracle.c).
"""
from __future__ import annotations

import numpy as np

NIN, NH = 5, 64
OFF_W1, OFF_B1 = 0, 320
OFF_W2, OFF_B2 = 384, 4480
OFF_W3, OFF_B3 = 4544, 4608
NPARAMS = 4609
MASK = (1 << 64) - 1


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[OFF_W1:OFF_B1].reshape(NH, NIN), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(NH, NH),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3], p[OFF_B3])


def forward(p, x):
    """y[n] for features x[n, 5] (FP64)."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    h1 = np.tanh(x @ W1.T + b1)
    h2 = np.tanh(h1 @ W2.T + b2)
    return h2 @ W3 + b3


def loss_and_grad(p, x, t):
    """Mean squared error over the samples and its gradient (FP64)."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    x = np.asarray(x, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    n = len(t)
    h1 = np.tanh(x @ W1.T + b1)
    h2 = np.tanh(h1 @ W2.T + b2)
    y = h2 @ W3 + b3
    e = 2.0 * (y - t) / n
    g = np.zeros(NPARAMS)
    g[OFF_B3] = e.sum()
    g[OFF_W3:OFF_B3] = h2.T @ e
    dz2 = (e[:, None] * W3[None, :]) * (1.0 - h2 * h2)
    g[OFF_B2:OFF_W3] = dz2.sum(0)
    g[OFF_W2:OFF_B2] = (dz2.T @ h1).reshape(-1)
    dz1 = (dz2 @ W2) * (1.0 - h1 * h1)
    g[OFF_B1:OFF_W2] = dz1.sum(0)
    g[OFF_W1:OFF_B1] = (dz1.T @ x).reshape(-1)
    return float(np.mean((y - t) ** 2)), g


def features(norm, d, rhop, psi, rhoa, mu):
    """Feature rows and the output constant ln(g d^2 rhop K1/18) per point;
    norm = the 19 numbers of f3d_mlp_get_norm."""
    lar_c, lar_sinv, sg_scale, psi_lo, psi_sinv, lnd_lo, lnd_sinv, lnmu_lo, lnmu_sinv = norm[:9]
    d, rhop, psi, rhoa, mu = (np.asarray(a, dtype=np.float64) for a in (d, rhop, psi, rhoa, mu))
    lnd, lnmu = np.log(d), np.log(mu)
    lar = np.log(9.81) + 3.0 * lnd + np.log(rhop) + np.log(rhoa) - 2.0 * lnmu
    sg = np.power(-np.log10(psi), 0.5743)
    f = np.stack([(lar - lar_c) * lar_sinv, sg * sg_scale - 1.0, (psi - psi_lo) * psi_sinv - 1.0,
                  (lnd - lnd_lo) * lnd_sinv - 1.0, (lnmu - lnmu_lo) * lnmu_sinv - 1.0], 1)
    k1 = 3.0 / (1.0 + 2.0 / np.sqrt(psi))
    cout = np.log(9.81) + 2.0 * lnd + np.log(rhop) + np.log(k1) - np.log(18.0)
    return f, cout


def target(cout, v, mu):
    """y = (ln Re - ln(Ar K1/18)) / 4 = (ln v - cout + ln mu) / 4."""
    return 0.25 * (np.log(v) - cout + np.log(mu))


def velocity(y, cout, mu):
    return np.exp(4.0 * y + cout - np.log(mu))


def predict(p, norm, d, rhop, psi, rhoa, mu):
    f, cout = features(norm, d, rhop, psi, rhoa, mu)
    return velocity(forward(p, f), cout, mu)


def _mix64(z):
    z = (z + 0x9E3779B97F4A7C15) & MASK
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
    return z ^ (z >> 31)


def hash3(seed, a, b):
    return _mix64(_mix64(_mix64(seed) ^ a) ^ ((b * 0xD1B54A32D192ED03) & MASK))


def draw_samples(seed, first, n, box):
    """The raw (d, rhop, psi, rhoa, mu) of samples first..first+n-1 drawn over
    box = [(lo, hi)] * 5 (the training box): diameter log-uniform, the
    others uniform."""
    out = np.empty((n, 5))
    for r in range(n):
        q = first + r
        for c in range(5):
            u = (hash3(seed, q, c) >> 11) * 2.0 ** -53
            lo, hi = box[c]
            if c == 0:
                out[r, c] = np.exp(np.log(lo) + u * (np.log(hi) - np.log(lo)))
            else:
                out[r, c] = lo + u * (hi - lo)
    return out
