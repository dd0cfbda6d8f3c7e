"""StreamCompact (StreamCompact.pyx:22-82) on libgcut; see IncrementalTileList.py."""
from IncrementalTileList import StreamCompact  # noqa: F401
