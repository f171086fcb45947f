"""witwin_channel_b200: B200-native deterministic radiomap/path engine.

Drop-in for ``witwin.channel.deterministic`` (``Config``, ``PathTable``,
``Result``, ``solve``) backed by hand-written sm_100a CUDA kernels in
``csrc/libwcb200.so`` reached through a plain C ABI.
"""

from . import constants, scene
from .deterministic import Config, PathTable, Result, solve

__all__ = ["Config", "PathTable", "Result", "constants", "scene", "solve"]
