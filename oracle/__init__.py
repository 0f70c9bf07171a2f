"""Oracle for incrmt_b200's parity tests.

TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference legs may import this package; the
product (incrmt_b200) never does.

Contents:
  - tgmg_shim/: clean-room restatement of the absent TGMG multigrid library
    behind the API the reference calls;
  - harness/ + Makefile: the reference's own sources compiled unmodified with
    that shim into _ref/libincrmt_ref.so (and _ref/ref_run);
  - refsim.py: ctypes access to _ref/libincrmt_ref.so;
  - operators.py: numpy restatement of the two pressure operators, an
    independent residual check.
"""
