"""riggle_b200 — B200 (sm_100a) implementation of chuckle's file-to-file interval-sweep hot path.

The product is libriggle_b200.so (C ABI in include/riggle.h); this package is its Python face.
"""
from ._lib import RiggleError, load, LIB_PATH  # noqa: F401
from .api import (  # noqa: F401
    CHROM_NAMES_24,
    BedBatch,
    Context,
    DeviceBatch,
    Index,
    LayerConfig,
    Server,
    SynthSpec,
    bucket_layers,
    synth_batch_device,
    synth_batch_layout,
    synth_chrom_lengths,
    synth_loguniform_sizes,
    synth_zipf_sizes,
)
