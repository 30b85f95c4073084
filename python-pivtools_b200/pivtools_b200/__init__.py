"""pivtools_b200 -- B200-native (sm_100a) PIVtools correlation hot path.

Drop-in CUDA implementations of libbulkxcorr2d, libfusedwarp and libkspacefit
(same C symbols and array layouts), plus resident-GPU drivers for multipass,
ensemble and served PIV.
"""

from . import geometry  # noqa: F401

__all__ = ["geometry"]
