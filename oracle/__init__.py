"""CPU oracle for the HOS hot path (test infrastructure only).

``ref_c`` drives the reference's own Csource/2dpar hot-path sources built
against a single-rank FFTW-MPI shim (oracle/Makefile); ``hos_np`` is an
independent numpy restatement.  Only tests/, the smoke check and the
bench's CPU baseline leg use this package.
"""
