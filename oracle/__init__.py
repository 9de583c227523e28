"""CPU checker for the QBX-FMM apply.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may import this package; the product
(``pytential_b200``) never does.
"""
