"""TEST INFRASTRUCTURE ONLY: CPU restatements of the reference algorithms (the checker).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use this package.
"""
