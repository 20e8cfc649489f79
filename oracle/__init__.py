"""Test infrastructure: CPU restatement of the reference algorithm (the oracle).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
package, as a checker; the product (ngap_b200) never imports it.
"""
