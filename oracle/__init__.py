"""CPU ORACLE for the DFSPH time step — test infrastructure only.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs may import this
package, and only as the checker or the timed CPU baseline: the product (splishsplash_for_cuda_b200)
never calls it and has no CPU fallback.

dfsph_oracle.cpp restates the reference GPU formulation of the step on the CPU (file:line citations
in its header). Parity pins: the kernel function is compared against the reference's own
CubicKernelPerso compiled from its header (ref_harness/), the neighbour sets against the
reference's ITER_NEIGHBORS macro run on the host, and the density / alpha fields against the
reference CPU solver TimeStepDFSPH (see tests/test_oracle_pins.py). The reference ships no golden
vectors or tests of its own.
"""
from .oracle import Oracle, OracleParams, build, lib_path  # noqa: F401
