"""Array helpers (vamtoolbox.util counterpart)."""
from . import data
