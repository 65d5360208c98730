"""Measurement drivers behind the figures under profiles/ (not part of the
importable library): run from the repository root as
``python -m benchmarks.<name>``."""
