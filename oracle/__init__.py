"""Oracle: CPU restatement of TigerCI's sigma-build path (test infrastructure
only).  Imported by tests/, __graft_entry__.smoke() and the CPU-baseline leg of
bench.py; never by the product package."""
