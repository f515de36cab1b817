"""The oracle: CPU restatements of exafmm-t used as the checker by the tests,
``__graft_entry__.smoke`` and the CPU-baseline leg of ``bench.py``.  Test
infrastructure only -- the product (exafmm-t_b200/) never imports it."""
