"""Python view of libvidstab_b200: vid.stab's motion-detection pass on a B200.

The product is the C library (include/vidstab_b200.h); this package only
binds it for tests, benchmarks and Python callers.
"""
from ._lib import (LM_DTYPE, TRANSFORM_DTYPE, PF_BGR24, PF_GRAY8, PF_RGB24, PF_RGBA, PF_YUV420P, PF_YUVA420P,
                   ASCII_SERIALIZATION_MODE, BINARY_SERIALIZATION_MODE, lib)
from .api import (Batch, MotionDetector, detect_clip, detect_multi, boxblur, boxblur_tile,
                  field_minmax, field_search, bpp_of, motions_to_transforms)

__all__ = ["LM_DTYPE", "PF_GRAY8", "PF_YUV420P", "PF_YUVA420P", "PF_RGB24", "PF_BGR24", "PF_RGBA",
           "ASCII_SERIALIZATION_MODE", "BINARY_SERIALIZATION_MODE", "lib", "Batch", "MotionDetector",
           "detect_clip", "detect_multi", "boxblur", "boxblur_tile", "field_minmax", "field_search",
           "bpp_of", "TRANSFORM_DTYPE", "motions_to_transforms"]
