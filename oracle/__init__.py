"""CPU FP64 oracle for the TEMF3DT FETD forward hot path.

TEST INFRASTRUCTURE ONLY.  Nothing in the shipped package imports this
directory; only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` use it, and only as the checker / the timed CPU
restatement.  See ``oracle/fetd_oracle.py`` for the restatement itself.
"""
