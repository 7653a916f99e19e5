"""The unmodified Chili reference (oracle/_ref) behind the shared oracle binding.

TEST INFRASTRUCTURE ONLY.
"""
from functools import partial

from .binding import REF, MultiChannel as _MC, am_adapt, am_map, am_split, am_weight, construct_channels, select, vegas_iterate, vegas_run  # noqa: F401


def available():
    return REF.available()


MultiChannel = partial(_MC, oracle=REF)
