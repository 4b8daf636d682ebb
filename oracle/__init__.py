"""TEST INFRASTRUCTURE: the CPU oracle (only tests, the smoke check and the
benchmark's CPU-baseline leg use it)."""
