"""CPU oracle — TEST INFRASTRUCTURE ONLY.

Restatements of the reference's algorithms (Peuqui/SolarSystemSimulator,
backend/*.py) on the CPU, each function citing the reference file:line it
follows. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
legs may import this package; the product package never does.

Pinned by tests/test_oracle_golden.py against fixtures in tests/golden/,
which tests/golden/make_golden.py generated by running the reference's own
NumPy code (through a cupy->numpy import shim) in the build container.
"""
