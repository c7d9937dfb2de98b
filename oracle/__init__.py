"""Oracle package: CPU restatement of the reference single-street solver and
loaders for the reference builds.  TEST INFRASTRUCTURE ONLY -- imported by
tests/, the smoke check and bench.py's CPU baseline, never by the product."""
