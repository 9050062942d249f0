"""CPU oracle for the NEGF hot path -- TEST INFRASTRUCTURE, never the product.

This package restates the reference algorithms in numpy (complex128) so the
CUDA path can be checked against them.  Only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` may import it, and only as the checker or the timed CPU
baseline.  The product package ``dpnegf_b200`` never imports it and has no CPU
fallback.

Parity of the restatement itself is pinned against fixtures produced by the
reference implementation (``tests/golden/make_golden.py`` runs the reference's
own ``recursive_gf``, ``surface_green``/``selfEnergy``, ``DeviceProperty``
trace routines, ``ozaki_residues`` and ``gauss_xw`` on seeded inputs).
"""
