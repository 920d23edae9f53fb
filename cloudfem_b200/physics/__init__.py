"""Drop-in replacements of cloudfem.physics (3D elasticity, A-V blocks)."""
