"""B200 polar Fourier correlation search (SIMPLE 3.0 polarft_corrcalc drop-in).

The directory name contains a dot, so import it through ``load_package()`` in
``__graft_entry__`` (which registers it as ``simple3_0_b200``)."""
from . import batching, build, shard, synth  # noqa: F401
from ._lib import load as load_library  # noqa: F401
from .pftcc import PftccError, ctfparams_array, polarft_corrcalc  # noqa: F401
