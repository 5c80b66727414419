"""CPU oracle for the pseudo-spectral nonlinear stage — TEST INFRASTRUCTURE ONLY.

This package restates, in plain numpy FP64, the reference algorithms that the
CUDA path in ``magic_b200`` replaces:

* ``oracle.grid``      Gauss-Legendre grid, lm maps, associated-Legendre tables
                       (reference ``horizontal_data.py``, ``blocking.py``,
                       ``plms.py``, ``params.py``)
* ``oracle.sht``       scalar and toroidal/poloidal transforms in both directions
                       (reference ``sht.py``)
* ``oracle.nonlinear`` grid-space products and the Courant reduction
                       (reference ``get_nl.py``, ``get_nl_anel.py``, ``courant.py``)

It is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may import it.
The product path (``magic_b200``) never imports it and fails loudly when its
CUDA library is missing.

Parity pin: the oracle is checked against golden vectors produced by running
the reference itself (``tests/golden/make_golden.py``, fixtures in
``tests/golden/*.npz``); see ``tests/test_oracle_golden.py``.
"""
