"""B200-native Kilosort4 template matching (run_matching / extract drop-in).

The compute path is the sm_100a library ``lib/libks_b200.so`` (C ABI in
``include/ks_b200.h``); this package is its host side.
"""
from .template_matching import (  # noqa: F401
    extract,
    install,
    peel,
    prepare_extract,
    prepare_matching,
    project_scores,
    run_matching,
    set_default_projection,
    spike_features,
    template_energy,
    transpose_ctc,
)

__version__ = "0.1.0"
