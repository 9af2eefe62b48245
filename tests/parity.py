"""Comparison helpers of the parity tests (oracle/compare.py)."""
from oracle.compare import *  # noqa: F401,F403
from oracle.compare import compare_counts, compare_event  # noqa: F401
