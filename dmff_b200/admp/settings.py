"""Default thresholds of the reference's fixed-step induced-dipole iteration (dmff/admp/settings.py)."""
POL_CONV = 1.0  # stop when max |dE/dU| over polarizable sites falls below this
MAX_N_POL = 30  # iteration limit
