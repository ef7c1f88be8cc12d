"""B200-native block-Wiedemann sequence engine over GF(p).

Drop-in replacement of the GPU stages of wilthoma/prym_green_ancillary
(cuda/cuprym_cyclic.cu and friends): hand-written sm_100a kernels behind the C
ABI in include/bw_engine.h, C++ drop-in executables under bin/, and this
ctypes binding for Python callers.
"""
from .engine import (  # noqa: F401
    EngineError,
    FORM_INT8,
    FORM_PLAIN,
    KoszulBatch,
    KoszulEngine,
    CyclicEngine,
    read_text,
    load,
    seeded_fill_device,
    seeded_fill_host,
)

TAG_MAPS, TAG_DIAG, TAG_X, TAG_Y = 1, 2, 3, 4
