"""TEST INFRASTRUCTURE ONLY: CPU oracles for the negacyclic multiplier.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this
package, and only as the checker (or the timed CPU port of the reference method).
The product path never imports it.
"""
