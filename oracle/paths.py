"""Where the reference source tree lies on the machine that builds the oracle.

One environment variable, PGX_REFERENCE, names the ParGeMSLR directory of the
reference checkout (the one holding INC/, SRC/ and TESTS/); the default is
the build container's mount.  Test infrastructure only: the product package
never reads the reference tree.
"""
import os

REFERENCE = os.environ.get("PGX_REFERENCE", "/root/reference/ParGeMSLR")
REFERENCE_TESTS = os.path.join(REFERENCE, "TESTS")
