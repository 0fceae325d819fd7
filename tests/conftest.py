"""Test configuration: registers the `gpu` marker and puts the package, the
oracle bindings and tests/ on sys.path."""
import os
import sys

# The CPU checkers link OpenBLAS and parallelise over boxes with OpenMP: one
# BLAS thread each (set before any checker library loads), or the two thread
# pools oversubscribe the cores (70x slower on the 65,536-dof workload).
os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "kern-interp-old_b200"), os.path.join(ROOT, "oracle"),
          os.path.dirname(os.path.abspath(__file__))):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
