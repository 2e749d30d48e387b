"""ORACLE — test infrastructure only.

CPU restatement of the reference's per-step Deep Potential evaluation
(model.py), neighbour list (nlist.py), MD updates (integrators.py) and the
shared Philox noise stream (philox.py).  Only tests/, __graft_entry__.smoke()
and bench.py's cpu_baseline / reference legs import it, and only as the
checker or the timed CPU baseline; the product never routes through it.
"""
