"""B200 implementation of the tjsq SU(2) t-J DMRG hot path.

libtjb200.so (built from csrc/ by build.py) implements model_wave + hmerge,
lanczos_memo_new, the reduced-density-matrix truncation and the correlator
contractions of DongNingSheng/Grand_SQL_tJ behind the C ABI of
include/tj_b200.h.  `lib` is the Python mirror of that interface; `synth`
and `lattice` build the inputs of the tests and the benchmark.
"""
