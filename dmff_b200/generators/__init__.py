"""Generator registry: importing this package registers every force-field generator by XML tag."""
from . import admp, classical, disp  # noqa: F401
