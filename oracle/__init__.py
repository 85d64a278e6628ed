"""CPU oracle for the Lippmann-Schwinger hot path (test infrastructure, not product).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
import this package. The product path (``jaxmaterials_b200``) never calls it.
"""
