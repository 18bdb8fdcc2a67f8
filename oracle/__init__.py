"""CPU oracle and reference harness for the Barnes-Hut engine.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the engine.
"""
