"""CPU oracle of the GCtfFind CTF path (test infrastructure only)."""
