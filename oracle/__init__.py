"""CPU oracle of WEST's Wstat response path: test infrastructure only.

Imported by tests/, __graft_entry__.smoke() and the CPU-baseline leg of
bench.py, and never by the west_b200 package.
"""
