"""Optimizers (vamtoolbox.optimizer counterpart): CAL, OSMO, BCLP, PM, FBP."""
from . import BCLP, CAL, FBP, OSMO, PM
