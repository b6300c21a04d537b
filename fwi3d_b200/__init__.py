"""fwi3d_b200 -- B200-native wave-propagation hot path of FWI3D.

The compute path is libfwi3d.so (hand-written sm_100a CUDA behind the C ABI in
include/fwi3d.h); `lib.Context` is its Python binding and `synth` builds the
seeded synthetic workloads.  Build with `python -m fwi3d_b200.build`.
"""
from . import lib, synth  # noqa: F401  (lib loads the .so only on first use)

__all__ = ["lib", "synth"]
