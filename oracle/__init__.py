"""CPU oracle of the reference's gate-application path — test infrastructure.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it, as
the checker; the engine in qoa_b200/ never imports it.
"""
