"""``funtable`` stand-in (no-op key/value store)."""
