"""``pacman.execspaces`` selector constants (src/common/execspaces.hpp:17-24).

Every selector is accepted and runs on the B200 engine; ``available()`` lists
all of them because none of them is backed by a different code path.
"""
SERIAL = 0x00
OPENMP = 0x01
THREADS = 0x02
CUDA = 0x03
HIP = 0x04
SYCL = 0x05

_VALID = {SERIAL, OPENMP, THREADS, CUDA, HIP, SYCL}


def available():
    """Names of the accepted execution-space selectors."""
    return ["SERIAL", "OPENMP", "THREADS", "CUDA", "HIP", "SYCL"]
