"""Oracle (test infrastructure only): checkers for the transport path.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
package.  ``refharness`` drives the reference's own traversal code compiled
for the host (oracle/_ref/libkpref_p{1,2}.so); ``port`` drives the C
restatement (oracle/_ref/libkporacle.so).
"""
