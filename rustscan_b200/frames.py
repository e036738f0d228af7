"""Frame hand-off: decoded 8-bit frames in pinned host memory, ready for the
device-side target conversion (RustGS/src/training/data/frame_targets.rs).

The reference converts each decoded frame to f32 on the host
(resize_rgb_u8_to_f32, frame_targets.rs:44-62) and uploads the f32 image
every step (engine/trainer.rs:94-107, 265-268). Here a decoded frame stays
bytes in pinned memory; Trainer.train_step_frames copies the bytes (a
quarter of the f32 volume) on a side stream while the previous step runs,
and gsr_frames_to_targets converts them on the device. Decoding, frame
order and caching stay with the caller's loader.
"""
from __future__ import annotations

import numpy as np


class FrameLoadError(RuntimeError):
    pass


class DecodedFrame:
    """One decoded frame: [height, width, 3] RGB bytes in pinned host memory
    (the `color_u8` of the reference's DecodedFrame)."""

    def __init__(self, rgb):
        import torch

        a = np.ascontiguousarray(rgb, dtype=np.uint8)
        if a.ndim != 3 or a.shape[2] != 3:
            raise FrameLoadError(f"decoded frame must be [height, width, 3] bytes, got shape {a.shape}")
        self.height, self.width = int(a.shape[0]), int(a.shape[1])
        self.rgb = torch.from_numpy(a).pin_memory() if torch.cuda.is_available() else torch.from_numpy(a)
