"""Solver-neutral propagation boundary (``witwin.channel.propagation``)."""

from . import consumer

__all__ = ["consumer"]
