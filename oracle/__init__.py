"""The oracle: CPU checkers for the B200 path (test infrastructure only).

Two independent CPU implementations of the reference's trace-and-optimise algorithm:

  * ``port``      -- liboracle.so, a plain-C restatement (mko_oracle.c) that cites the
                     reference file:line it follows for every function;
  * ``reference`` -- _ref/libmko_ref.so, the reference's own CPU sources compiled where they
                     lie by oracle/Makefile (present only where the reference tree was).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline legs import this
package; the product path (mikroptim_b200) never does.
"""

from .pyoracle import Port, Reference, build, port, reference  # noqa: F401
