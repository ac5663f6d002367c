"""ORACLE - test infrastructure only (tests/, smoke() and bench.py's CPU leg).

ctypes bindings to the plain-C restatement (liboracle.so, built from
spk_oracle.c by oracle/Makefile) and, where it was built, to the reference's
own C++ (oracle/_ref/libspk_ref.so, built by oracle/ref/Makefile).  The
product path never imports this package.
"""
