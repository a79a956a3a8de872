"""Choosing the device (mirrors chadmv/plume src/plume/sim/device.py:8-21).

This implementation runs every kernel on CUDA; asking for the CPU is an error rather than a silent fallback.
"""

import torch

DEVICE_CHOICES = ("auto", "cuda")


class DeviceError(Exception):
    """The requested device is not available."""


def init_device(choice: str = "auto") -> str:
    if choice == "cpu":
        raise DeviceError("plume_b200 runs its kernels on CUDA only; there is no CPU device")
    if not torch.cuda.is_available():
        raise DeviceError(f"--device {choice} was asked for, but no CUDA GPU is available")
    from plume_b200 import _native

    _native.lib()  # fail here, loudly, when the library is missing
    return "cuda:0"
