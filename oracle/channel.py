"""CFR of path records, FP64 (test infrastructure only).

Restates ``PathResult.cfr`` (``witwin/channel/path.py:646-656``): per link,
delays minus the link's smallest delay (``_masked_min``, ``path.py:340-350``)
when normalising, and H(f_k) = sum_p a_p exp(-j 2 pi tau_p f_k).
"""

from __future__ import annotations

import numpy as np


def cfr(tx, rx, tau, a, frequencies, num_tx: int, num_rx: int, normalize: bool = True) -> np.ndarray:
    tx = np.asarray(tx, dtype=np.int64)
    rx = np.asarray(rx, dtype=np.int64)
    tau = np.asarray(tau, dtype=np.float64)
    a = np.asarray(a, dtype=np.complex128)
    f = np.asarray(frequencies, dtype=np.float64)
    out = np.zeros((num_tx, num_rx, f.shape[0]), dtype=np.complex128)
    for t in range(num_tx):
        for r in range(num_rx):
            m = (tx == t) & (rx == r)
            if not m.any():
                continue
            tt = tau[m] - (tau[m].min() if normalize else 0.0)
            out[t, r] = (a[m][:, None] * np.exp(-2j * np.pi * tt[:, None] * f[None, :])).sum(axis=0)
    return out
