"""B200-native GCtfFind CTF-estimation path.

The compute lives in ``lib/libgctf_b200.so`` (hand-written sm_100a CUDA
behind the C ABI in ``include/gctf_b200.h``); :mod:`gctffind_b200.api`
mirrors the reference's CFindCtf2D / CCTFTheory interface over it, and
``bin/GCtfFind`` is the drop-in command line.
"""
from .api import (  # noqa: F401
    CCTFTheory, CFindCtf2D, Context, CtfParam, GcfError, Item, Optics, Result, GCF_SPECT_CUFFT,
    GCF_SPECT_FUSED, EXPORTS, LIB_PATH, CLI_PATH, load_library, make_optics, mrc_info, mrc_read,
    mrc_read_tilts, mrc_write, rescale_dims, series_order, write_ctf_file,
    GCF_SEARCH_PLAIN, GCF_SEARCH_BF16, GCF_SEARCH_LEARNED, GCF_RESCALE_LINES, GCF_RESCALE_CUFFT, GCF_RESCALE_GEMM,
)
from .learned import WEIGHTS_PATH, learned_available, load_learned  # noqa: F401
