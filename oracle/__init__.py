"""Test infrastructure: FP64 CPU oracle (oracle.py / oracle.cpp) and the
reference-build harness (ref.py / ref_harness.cu).  Never imported by the
product path."""
