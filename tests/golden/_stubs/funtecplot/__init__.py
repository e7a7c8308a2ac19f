"""``funtecplot`` stand-in (Tecplot writer is never called on the step path)."""
