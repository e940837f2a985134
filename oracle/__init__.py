"""FP64 CPU oracle for the RKS hot path (test infrastructure).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use this
package, and only as the checker or the timed CPU baseline; the product path never imports
it.  Modules:

* ``eri``  -- s8 unique ERIs: the C restatement (eri_oracle.c) and the reference's own
  compiled ``int2e_sph`` (oracle/_ref, built by build_ref.py from the reference sources).
* ``rks``  -- numpy FP64 restatement of the SCF: AO values on the grid, B3LYP
  (exchange_correlation/*.py), J/K (nanoDFT.py:125-139), DIIS (nanoDFT.py:338-364) and the
  iteration (nanoDFT.py:40-102), energies (nanoDFT.py:20-38).
"""
