"""The C restatement (oracle/port/chili_oracle.c) behind the shared oracle binding.

TEST INFRASTRUCTURE ONLY.
"""
from functools import partial

from . import binding
from .binding import PORT

am_map = partial(binding.am_map, oracle=PORT)
am_weight = partial(binding.am_weight, oracle=PORT)
am_adapt = partial(binding.am_adapt, oracle=PORT)
am_split = partial(binding.am_split, oracle=PORT)
vegas_iterate = partial(binding.vegas_iterate, oracle=PORT)
select = partial(binding.select, oracle=PORT)
philox_uniforms = partial(binding.philox_uniforms, oracle=PORT)
philox_stream_uniforms = partial(binding.philox_stream_uniforms, oracle=PORT)
MultiChannel = partial(binding.MultiChannel, oracle=PORT)


def available():
    return PORT.available()
