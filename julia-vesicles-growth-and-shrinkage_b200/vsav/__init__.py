"""B200-native pseudo-spectral SAV vesicle step (host side of libvsav)."""
from .core import Handle, VsavError, WCNegativeError, NotConvergedWarning  # noqa: F401
from . import ics  # noqa: F401
