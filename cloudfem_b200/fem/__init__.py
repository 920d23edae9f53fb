"""Drop-in replacements of cloudfem.fem (P1 and Tet10 scalar problems)."""
