"""td16_b200: B200-native witness search for the td16 emitter.

The product is the native library libtd16b200.so (C ABI in include/td16_b200.h);
this package binds it (``_lib``) and mirrors the reference's Java host model
for the search (``host``).
"""
from . import _lib  # noqa: F401
from ._lib import (INSTANCE_DTYPE, RESULT_DTYPE, TdError, init_slots, destroy, search,  # noqa: F401
                   search_batch, prepare_pairs, prepare_perms, synth_perms, unpack_moves)
from .host import GPUSortingSearch, GpuDeviceLayout, GpuSearchStats, PairBatcher  # noqa: F401
