"""Empty stand-in so the reference's I/O module imports (test infrastructure only)."""
