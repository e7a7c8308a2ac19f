"""``funvtk`` stand-in (VTK writers are never called on the step path)."""
