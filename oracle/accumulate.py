"""Flat per-cell accumulation, bit-exact restatement (test infrastructure only).

Follows ``native/channel/kernels/deterministic.cu:829-970`` (slot map, six
materialised slots, the coherent/incoherent finalisation) behind
``witwin/channel/kernels/deterministic.py:23-102``.  Sums run in path index
order in the requested precision, one IEEE rounding per add; the per-cell
coherent power is ``fma(re, re, im * im)`` (one rounding of the exact
``re * re + round(im * im)``), the form that reproduces the reference's frozen
SHA-256 outputs (``tests/ad/test_deterministic_accum_ad.py:42-62``).
"""

from __future__ import annotations

from fractions import Fraction

import numpy as np

SLOTS = 6
SCATTERING_SLOT = 4
COUPLED_SLOT = 5


def accum_slot(component_id: int) -> int:
    """``deterministic.cu:829-843``."""
    if 0 <= component_id < 3:
        return component_id
    if component_id in (3, 4, 7):
        return COUPLED_SLOT
    if component_id == 5:
        return 3
    if component_id == 6:
        return SCATTERING_SLOT
    return -1


def _round_f32(x: Fraction) -> np.float32:
    """Correctly rounded (nearest, ties to even) float32 of an exact rational."""
    f = np.float32(float(x))  # float(x) is correctly rounded; fix a possible double rounding below
    if Fraction(float(f)) == x or not np.isfinite(f):
        return f
    lo = f if Fraction(float(f)) < x else np.nextafter(f, np.float32(-np.inf))
    hi = np.nextafter(lo, np.float32(np.inf))
    dl, dh = x - Fraction(float(lo)), Fraction(float(hi)) - x
    if dl < dh:
        return lo
    if dh < dl:
        return hi
    return lo if (int(lo.view(np.uint32)) & 1) == 0 else hi


def fma(a, b, c, dtype):
    """Single-rounding a*b + c in ``dtype`` (float32 or float64)."""
    exact = Fraction(float(a)) * Fraction(float(b)) + Fraction(float(c))
    if dtype == np.float32:
        return _round_f32(exact)
    return np.float64(float(exact))


def cabs2(re, im, dtype):
    return fma(re, re, dtype(im * im), dtype)


def accumulate_flat(valid, tx_id, rx_id, component_id, path_gain, field_real, field_imag, *, num_tx: int,
                    num_rx: int, coherent: bool, scattering_coherent: bool = False, dtype=np.float32) -> dict:
    """Returns the reference's six outputs: power_total/field_total_* (T,R) and
    component_power/component_field_* (6,T,R), in ``dtype``."""
    dt = np.dtype(dtype).type
    cells = num_tx * num_rx
    P = np.zeros((SLOTS, cells), dt)
    Re = np.zeros((SLOTS, cells), dt)
    Im = np.zeros((SLOTS, cells), dt)
    g = np.asarray(path_gain).astype(dt)
    fr = np.asarray(field_real).astype(dt)
    fi = np.asarray(field_imag).astype(dt)
    for i in range(len(tx_id)):
        if not bool(valid[i]):
            continue
        s = accum_slot(int(component_id[i]))
        t, r = int(tx_id[i]), int(rx_id[i])
        if s < 0 or t < 0 or r < 0 or t >= num_tx or r >= num_rx:
            continue
        c = t * num_rx + r
        P[s, c] = dt(P[s, c] + g[i])
        Re[s, c] = dt(Re[s, c] + fr[i])
        Im[s, c] = dt(Im[s, c] + fi[i])
    pt = np.zeros(cells, dt)
    ftr = np.zeros(cells, dt)
    fti = np.zeros(cells, dt)
    for c in range(cells):
        rs = is_ = ps = sp = dt(0)
        for s in range(SLOTS):
            re, im = Re[s, c], Im[s, c]
            if coherent:
                if s == SCATTERING_SLOT:
                    if scattering_coherent:
                        P[s, c] = cabs2(re, im, dt)
                    sp = dt(sp + P[s, c])
                    continue
                P[s, c] = cabs2(re, im, dt)
            else:
                if s == SCATTERING_SLOT and scattering_coherent:
                    P[s, c] = cabs2(re, im, dt)
                ps = dt(ps + P[s, c])
            rs = dt(rs + re)
            is_ = dt(is_ + im)
        if coherent:
            ftr[c], fti[c] = rs, is_
            pt[c] = dt(cabs2(rs, is_, dt) + sp)
        else:
            pt[c] = ps
            ftr[c] = dt(np.sqrt(max(ps, dt(0))))
            fti[c] = dt(0)
    T, R = num_tx, num_rx
    return {
        "power_total": pt.reshape(T, R),
        "field_total_real": ftr.reshape(T, R),
        "field_total_imag": fti.reshape(T, R),
        "component_power": P.reshape(SLOTS, T, R),
        "component_field_real": Re.reshape(SLOTS, T, R),
        "component_field_imag": Im.reshape(SLOTS, T, R),
    }
