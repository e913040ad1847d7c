"""CPU oracle for the split-explicit ARW RK3 dycore step -- TEST INFRASTRUCTURE ONLY.

This package restates, in plain NumPy float64, the algorithm of wrf_gpu's
``_rk_scan_step`` (``src/gpuwrf/runtime/operational_mode.py:3319-3534``) and
every operator it calls on the flux-advection path.  Each function cites the
reference file:line it follows.

It is the checker, never the product: only ``tests/``, ``__graft_entry__.smoke``
and ``bench.py``'s CPU-baseline leg may import it.  The shipped path
(``wrf_gpu_b200``) runs hand-written CUDA and fails loudly when its extension
is missing; it never routes through this package.

Parity pinning.  The reference is pure JAX and JAX is not installed where this
was written, so no outputs of the reference step itself could be generated.
The restatement is pinned against the reference's own known-answer tests for
this path, re-run here on the oracle:

* ``scripts/f7a_oracles.py:265-446`` -- flat rest state stays at rest (AC3),
  a +1 K layer gives an upward/downward w dipole and a geopotential rise (AC4),
  and a long pure-acoustic run conserves dry mass to 1e-6 (AC5);
* ``src/gpuwrf/ic_generators/idealized.py:751-773`` with
  ``tests/idealized/test_warm_bubble.py`` -- the 2-D Skamarock warm bubble gates
  at 500 s (0.5 <= theta'max <= 2.5 K, 1 <= max|w| <= 30 m/s, centroid rise
  >= 500 m, drift <= 250 m, relative dry-mass drift <= 1e-8), plus the
  reference's recorded gate values (``proofs/v040/idealized_no_regression_report.json``:
  max|w| 11.680 m/s, rise 1924.35 m, theta'max 1.9201 K) as a closeness check.

The gate values were recorded by older reference versions, so they pin the
algorithm to a tolerance, not bit-for-bit: parity of the CUDA path is
therefore measured against this restatement (1e-12 relative per field per
step), and this restatement against the reference's gates.
"""
