"""epb200: B200-native Wannier->Bloch electron-phonon interpolation (host-side mirror).

The compute path is the sm_100a shared library `libepb200.so` (C ABI, `include/epb200.h`).
This package mirrors the reference's Julia API for that path (WannierObject, batched eigensolves,
the list-batched e-ph drivers, rotations, window filter) on top of torch device buffers.
"""
from .wannier import WannierObject, to_device  # noqa: F401
