"""CPU oracle for the CPR-Krylov hot path — TEST INFRASTRUCTURE ONLY.

  oracle.port  numpy / C restatement of the reference's algorithms (deco_oracle.c),
               each function citing the reference file:line it follows;
  oracle.ref   the reference's own code compiled from its sources (oracle/ref/Makefile)
               behind single-rank MPI, ptree and LAPACKE-prototype shims.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs import this
package, and only as the checker or as the timed CPU baseline.
"""
