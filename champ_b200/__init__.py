"""champ_b200: walker-batched Slater-Jastrow engine (CHAMP hot path) for B200.

The compute path is the CUDA library ``libchamp_b200.so`` built in-tree from
``csrc/`` (see ``champ_b200.build``); this package only binds its C ABI.
There is no CPU fallback: loading fails loudly when the library is missing.
"""
from .engine import Engine, load_library, EXPORTED_SYMBOLS  # noqa: F401
from . import system  # noqa: F401
