"""Frame pipeline: the deterministic frame order, a prefetching decoded-frame
cache in pinned host memory, and the hand-off of 8-bit frames to the device
(RustGS/src/training/data/frame_loader.rs, frame_targets.rs).

The reference decodes frames on worker threads into RGB bytes, converts them
to f32 targets on the host and uploads the f32 image every step
(engine/trainer.rs:94-107, 265-268). Here decoded frames stay bytes in
pinned memory; the bytes cross PCIe (a quarter of the f32 volume) on a side
stream while the previous step runs, and gsr_frames_to_targets converts them
on the device (see Trainer.train_step_frames).
"""
from __future__ import annotations

import threading
from collections import OrderedDict
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass

import numpy as np

_MASK64 = (1 << 64) - 1
_GOLDEN = 0x9E3779B97F4A7C15  # SplitMix64 increment (Steele, Lea, Flood 2014)


class SplitMix64:
    """The SplitMix64 generator (frame_loader.rs:560-587): a Weyl sequence
    with the published 64-bit finaliser."""

    def __init__(self, seed: int):
        self.state = (seed + _GOLDEN) & _MASK64

    def next_u64(self) -> int:
        z = self.state
        self.state = (self.state + _GOLDEN) & _MASK64
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _MASK64
        return z ^ (z >> 31)

    def next_index(self, upper: int) -> int:
        return 0 if upper <= 1 else self.next_u64() % upper


def deterministic_shuffle(indices: list, seed: int) -> None:
    """In-place Fisher-Yates shuffle seeded with seed ^ (len << 32)
    (frame_loader.rs:589-595)."""
    rng = SplitMix64((seed ^ (len(indices) << 32)) & _MASK64)
    for i in range(len(indices) - 1, 0, -1):
        j = rng.next_index(i + 1)
        indices[i], indices[j] = indices[j], indices[i]


class DeterministicFrameBatchIter:
    """Frame indices in batches (frame_loader.rs:59-107): identity order for
    seed 0, else the seeded shuffle; the last batch may be short."""

    def __init__(self, frame_count: int, batch_size: int, seed: int):
        self._order = list(range(frame_count))
        if seed != 0:
            deterministic_shuffle(self._order, seed)
        self.batch_size = max(batch_size, 1)
        self._cursor = 0

    def order(self) -> list:
        return list(self._order)

    def __iter__(self):
        return self

    def __next__(self) -> list:
        if self._cursor >= len(self._order):
            raise StopIteration
        end = min(self._cursor + self.batch_size, len(self._order))
        batch = self._order[self._cursor:end]
        self._cursor = end
        return batch


def ordered_frame_indices(frame_count: int, batch_size: int, seed: int) -> list:
    """The batches of DeterministicFrameBatchIter, flattened (frame_loader.rs:84-92)."""
    return [i for b in DeterministicFrameBatchIter(frame_count, batch_size, seed) for i in b]


@dataclass
class FrameLoaderOptions:
    """frame_loader.rs:24-39."""
    cache_capacity: int = 8
    prefetch_ahead: int = 4


def frame_loader_worker_count(frame_count: int, options: FrameLoaderOptions, parallelism: int | None = None) -> int:
    """Decoding threads: at most the frames, the prefetch window and the host
    threads (frame_loader.rs:339-345)."""
    import os

    par = parallelism if parallelism is not None else (os.cpu_count() or 4)
    return min(max(frame_count, 1), max(options.prefetch_ahead, 1), max(par, 1))


class FrameLoadError(RuntimeError):
    pass


class DecodedFrame:
    """One decoded frame: [height, width, 3] RGB bytes in pinned host memory."""

    def __init__(self, rgb):
        import torch

        a = np.ascontiguousarray(rgb, dtype=np.uint8)
        if a.ndim != 3 or a.shape[2] != 3:
            raise FrameLoadError(f"decoded frame must be [height, width, 3] bytes, got shape {a.shape}")
        self.height, self.width = int(a.shape[0]), int(a.shape[1])
        self.rgb = torch.from_numpy(a).pin_memory() if torch.cuda.is_available() else torch.from_numpy(a)


class PrefetchFrameLoader:
    """Decoded-frame cache with background decoding (frame_loader.rs:109-337).

    decode(frame_idx) returns a [height, width, 3] uint8 array (the caller's
    image decoder: the reference uses the `image` crate). Worker threads
    decode the frames of the prefetch window; get() returns a cached frame or
    waits for it; the cache keeps the most recently used cache_capacity
    frames. A frame whose decoding failed raises when it is requested."""

    def __init__(self, decode, frame_count: int, options: FrameLoaderOptions | None = None):
        if frame_count <= 0:
            raise FrameLoadError("training dataset does not contain any poses")
        self.options = options or FrameLoaderOptions()
        self.frame_count = frame_count
        self._decode = decode
        self._cache: OrderedDict[int, DecodedFrame] = OrderedDict()
        self._pending: dict = {}
        self._lock = threading.Lock()
        self._pool = ThreadPoolExecutor(max_workers=frame_loader_worker_count(frame_count, self.options))

    def close(self):
        self._pool.shutdown(wait=True)

    def __del__(self):
        try:
            self._pool.shutdown(wait=False)
        except Exception:
            pass

    def _check(self, frame_idx: int):
        if not 0 <= frame_idx < self.frame_count:
            raise FrameLoadError(f"frame index {frame_idx} is outside the dataset bounds")

    def _queue(self, frame_idx: int):
        self._check(frame_idx)
        if frame_idx in self._cache or frame_idx in self._pending:
            return
        self._pending[frame_idx] = self._pool.submit(lambda i=frame_idx: DecodedFrame(self._decode(i)))

    def _insert(self, frame_idx: int, frame: DecodedFrame):
        self._cache[frame_idx] = frame
        self._cache.move_to_end(frame_idx)
        while len(self._cache) > max(self.options.cache_capacity, 1):
            self._cache.popitem(last=False)

    def _drain_ready(self):
        for idx in [i for i, f in self._pending.items() if f.done()]:
            fut = self._pending.pop(idx)
            try:
                frame = fut.result()
            except Exception as e:
                raise FrameLoadError(f"prefetch failed for frame {idx}: {e}") from e
            self._insert(idx, frame)

    def prefetch_order_window(self, order, cursor: int):
        """Queue the frames order[cursor : cursor + prefetch_ahead]."""
        for idx in order[cursor:min(cursor + self.options.prefetch_ahead, len(order))]:
            self._queue(idx)
        self._drain_ready()

    def get(self, frame_idx: int) -> DecodedFrame:
        self._check(frame_idx)
        self._drain_ready()
        if frame_idx in self._cache:
            self._cache.move_to_end(frame_idx)
            return self._cache[frame_idx]
        self._queue(frame_idx)
        fut = self._pending.pop(frame_idx)
        frame = fut.result()  # a decoding error of the requested frame propagates
        self._insert(frame_idx, frame)
        return frame

    def cache_len(self) -> int:
        return len(self._cache)

    def is_cached(self, frame_idx: int) -> bool:
        return frame_idx in self._cache
