"""Host side of the B200-native ISPH step (ctypes over include/sph_isph.h)."""
from . import layout, params, decks  # noqa: F401
