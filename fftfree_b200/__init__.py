"""fftfree_b200 -- the fftfree batched STFT/FFT hot path on NVIDIA B200.

The product is the C-ABI shared library ``lib/libfft_cffi.so`` (built from
``csrc/`` by ``build.py``); this package binds it (``api``) and adds the
torch-facing helpers.  See include/fft_cffi.h for the ABI.
"""
from .api import (  # noqa: F401
    EXPORTED,
    LIB_PATH,
    FftContext,
    MetadataRequest,
    RESTORE_OBSERVER,
    device_available,
    lib,
)
from .api import *  # noqa: F401,F403
