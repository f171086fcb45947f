"""FP64 CPU oracle for the deterministic radiomap/path hot path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product package imports this
directory; only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` use it, and only as the checker.

The oracle restates, in float64/complex128 NumPy, the algorithm of the
reference's deterministic solver (``witwin/channel/deterministic.py`` and the
modules it calls).  Each function cites the reference file:line it follows.
Where the reference delegates to its external ray-tracing library (RayD @
c7a99979, rayd-torch 0.8.0: image-method EPC, visibility, penetration, UTD),
the oracle restates the published algorithm (image method, watertight
segment/triangle tests, Kouyoumjian-Pathak UTD with the finite-edge rules of
the reference's ``docs/dev/audit/utd-continuity-fix-design.md`` F1-F5f) and is
pinned by the reference's own golden vectors (two-wall multibounce lengths and
sequences, the single-wedge edge ids and lengths, the closed-form free-space
and slab tests).  The UTD amplitudes are only partially pinned: the
reference's exact RayD assembly is not available.
"""
