"""Generator registry: importing this package registers the drop-in generator classes."""
from . import admp  # noqa: F401
from . import disp  # noqa: F401
