"""TEST INFRASTRUCTURE ONLY: the oracle (a CPU restatement of the reference
integrator) and the reference's own CPU code built from its sources.

Only tests, the smoke check and the benchmark's CPU-baseline leg import
this package, as the checker; the product never does.
"""
