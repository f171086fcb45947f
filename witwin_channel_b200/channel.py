"""Channel views of an exported path table: CIR, CFR and taps.

Same definitions as the reference's ``PathResult.cir`` / ``.cfr`` / ``.taps``
(``witwin/channel/path.py:637-700``), applied per (tx, rx) link of a
deterministic ``PathTable`` (records in canonical (rx, tx) order): delays are
normalised per link by their minimum, the coefficient is the powered path
field, and the CFR is H(f_k) = sum_p a_p exp(-j 2 pi tau_p f_k).  The CFR runs
in ``libwcb200.so`` (``wcb_cfr``), one warp per link, each link's spectrum
written once.
"""

from __future__ import annotations

import ctypes

import torch

from . import _native, engine

_CFR_WORKSPACE = engine.Workspace()


def _coefficients(paths) -> torch.Tensor:
    return torch.complex(paths.field_real.float(), paths.field_imag.float())


def cfr(paths, frequencies, *, num_tx: int, num_rx: int, normalize_delays: bool = True) -> torch.Tensor:
    """(num_tx, num_rx, K) complex64 frequency response at ``frequencies`` (Hz,
    shape (K,)).  An evenly spaced grid takes the rotation fast path."""
    if not isinstance(frequencies, torch.Tensor):
        frequencies = torch.as_tensor(frequencies, dtype=torch.float64)
    if frequencies.ndim != 1:
        raise ValueError("frequencies must have shape (frequency,)")
    K = int(frequencies.shape[0])
    if K < 1:
        raise ValueError("frequencies must not be empty")
    device = paths.tx_id.device
    freqs = frequencies.to(device=device, dtype=torch.float64).contiguous()
    f_host = freqs.cpu()
    df = 0.0
    if K > 1:
        steps = f_host[1:] - f_host[:-1]
        if float((steps - steps[0]).abs().max()) <= 1e-9 * max(float(steps[0].abs()), 1.0):
            df = float(steps[0])
    elif K == 1:
        df = 1.0  # a single subcarrier: any step works
    n = int(paths.tx_id.shape[0])
    if n > 1:
        key = paths.rx_id.long() * max(int(num_tx), 1) + paths.tx_id.long()
        if bool((key[1:] < key[:-1]).any()):
            raise ValueError("paths must be in the canonical (rx, tx) order of an exported path table")
    out = torch.empty((num_tx, num_rx, K), dtype=torch.complex64, device=device)
    a = _coefficients(paths).contiguous()
    lib = _native.load()
    nbytes = ctypes.c_int64()
    _native.check(lib.wcb_cfr_workspace_size(int(num_tx), int(num_rx), ctypes.byref(nbytes)), "wcb_cfr_workspace_size")
    ws = _CFR_WORKSPACE.get(nbytes.value, device)
    _native.check(
        lib.wcb_cfr(_native.ptr(paths.tx_id.contiguous()) if n else None,
                    _native.ptr(paths.rx_id.contiguous()) if n else None,
                    _native.ptr(paths.delay_s.float().contiguous()) if n else None,
                    _native.ptr(torch.view_as_real(a)) if n else None, n, int(num_tx), int(num_rx), K,
                    float(f_host[0]), df, _native.ptr(freqs), int(bool(normalize_delays)), _native.ptr(out),
                    _native.ptr(ws), ws.numel(), _native.stream_handle(device)),
        "wcb_cfr",
    )
    return out


def cir(paths, *, normalize_delays: bool = True) -> tuple[torch.Tensor, torch.Tensor]:
    """Per record: the complex coefficient and its delay (normalised per link
    when ``normalize_delays``)."""
    a = _coefficients(paths)
    tau = paths.delay_s.double()
    if normalize_delays and tau.numel():
        key = paths.tx_id.long() * (int(paths.rx_id.max()) + 1) + paths.rx_id.long()
        mins = torch.full((int(key.max()) + 1,), float("inf"), dtype=torch.float64, device=tau.device)
        mins = mins.scatter_reduce(0, key, tau, reduce="amin")
        tau = tau - mins[key]
    return a, tau.float()


def taps(paths, bandwidth: float, num_taps: int, *, num_tx: int, num_rx: int,
         normalize_delays: bool = True) -> torch.Tensor:
    """(num_tx, num_rx, num_taps) complex64: each record's coefficient added to
    tap round(tau * bandwidth) of its link (reference ``taps``, path.py:660-700)."""
    if bandwidth <= 0.0:
        raise ValueError("bandwidth must be > 0")
    if num_taps <= 0:
        raise ValueError("num_taps must be > 0")
    a, tau = cir(paths, normalize_delays=normalize_delays)
    out = torch.zeros((num_tx * num_rx * num_taps,), dtype=torch.complex64, device=a.device)
    if a.numel() == 0:
        return out.reshape(num_tx, num_rx, num_taps)
    tap = torch.round(tau.double() * float(bandwidth)).long()
    keep = (tap >= 0) & (tap < num_taps)
    idx = (paths.tx_id.long() * num_rx + paths.rx_id.long()) * num_taps + tap
    out.index_put_((idx[keep],), a[keep], accumulate=True)
    return out.reshape(num_tx, num_rx, num_taps)
