"""Oracle package — test infrastructure only (CPU restatement of the reference's algorithm).

Importable from tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm;
the product package (pyspectral_b200) never imports it.
"""
