"""Ray-march parameters (mirrors chadmv/plume src/plume/render/raymarch.py:21-52). The march itself is the
library's raymarch kernel, called by FrameRenderer.march."""

from plume_b200._native import PlumeLookParams as LookParams
from plume_b200._native import PlumeViewParams as ViewParams

FAR_M = 1.0e4

__all__ = ["FAR_M", "LookParams", "ViewParams"]
