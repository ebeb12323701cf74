"""CPU oracle of the reference's per-stage DG update (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs may import this package.  See
mhd_oracle.h for what it restates and for its parity status ("parity unpinned" against a run of
the reference, which cannot be compiled on this machine; pinned through the reference's own
known answers and invariants).
"""
