"""CPU oracle for the HOS hot path (test infrastructure only).

``ref_c`` drives the reference's own Csource/2dpar hot-path sources built
against a single-rank FFTW-MPI shim (oracle/Makefile); ``hos_np`` is an
independent numpy restatement.  Only tests/, the smoke check and the
bench's CPU baseline leg use this package.
"""

import os as _os

# The reference's Csource/2dpar directory (its hot-path sources and shipped
# inputs).  It exists only where the oracle is built; the environment
# variable HOS_REFERENCE_SRC moves it (oracle/Makefile reads the same one).
REFERENCE_SRC = _os.environ.get("HOS_REFERENCE_SRC", "/root/reference/Csource/2dpar")
