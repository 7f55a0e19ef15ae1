"""worldinagrain_b200: the liquid step of the falling-sand world on B200."""
from . import abi  # noqa: F401
