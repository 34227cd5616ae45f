"""Classical force-field terms (LJ, point-charge Coulomb, bonded) on the B200 engine."""
