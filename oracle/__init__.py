"""ORACLE: CPU restatement of the reference's alm2map path and the
reference's own C library (built by oracle/Makefile into oracle/_ref/),
used only as a checker by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg.  Nothing in the product imports this package."""
