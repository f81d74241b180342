"""The oracle: a CPU restatement of the reference's SN solve, used only as the checker by
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg."""
