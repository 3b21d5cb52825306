"""CPU oracle for the line-by-line transmittance path — TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package; the product (``pylblrtm_b200``) never
does. ``restate`` is a float64 NumPy/SciPy restatement of the reference forward
model (``pylblrtm/forward.py:41-317``, ``atmosphere.py:110-141``,
``spectral_data.py:43-52``); it is pinned against golden vectors produced by the
reference itself (``tests/golden/make_golden.py``).
"""
