"""B200-native implementation of FMT2D's forward-and-sensitivity path.

Eikonal time fields of every OBS source and phase stage, the ray backtrace,
Frechet rows and LSQR products, behind the C ABI of include/fmt2d_gpu.h.
"""
from .synth import SmeshModel, config, small_model  # noqa: F401


def api():
    """The context class (imported lazily: loading it loads the native library)."""
    from .api import Fmt2d
    return Fmt2d
