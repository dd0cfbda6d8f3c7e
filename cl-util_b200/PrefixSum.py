"""PrefixSum (PrefixSum.pyx:121-226) on libgcut; see IncrementalTileList.py."""
from IncrementalTileList import PrefixSum  # noqa: F401
