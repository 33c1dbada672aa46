"""CPU oracle for kascade_b200 -- TEST INFRASTRUCTURE ONLY.

Loads the plain-C restatement of the reference's algorithms
(oracle/kascade_oracle.c) and, when it was built from the reference source
tree, the reference's own GatherChase (oracle/_ref).  Only the tests, the
smoke entry and the bench's CPU-baseline leg use this package; the
kascade_b200 library never does.
"""
from .oracle import *  # noqa: F401,F403
