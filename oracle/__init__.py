"""Test infrastructure: the CPU oracle and the reference build.

Only tests, the smoke entry point and the bench's reference/CPU-baseline legs
use this package. REFROOT is where the reference's sources lie (the same
variable oracle/Makefile reads); it is needed only to build oracle/_ref and to
regenerate fixtures, never on a machine that runs the GPU tests.
"""
import os

REFROOT = os.environ.get("REFROOT", "/root/reference")
