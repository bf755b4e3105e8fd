"""Streaming CWT: overlapping windows of a long signal.

The reference's README advertises real-time use (a CWT of the latest window
of a live signal, README.md:27); its API transforms one buffer per call and
re-plans every time (FCWT::cwt, src/fcwt/fcwt.cpp:447-529). Here a window of
`window` samples slides by `hop` samples: the samples live in one device
buffer, the plan is built once, and every frame replays the same CUDA graph
(forward FFT + row kernels) on that buffer, so a frame costs one graph launch
and a shift of the buffer.

    s = StreamingCWT(window=16384, hop=4096, scales=sc, fb=2.0)
    for block in source:                 # numpy or torch CUDA, any length
        for frame in s.push(block):      # [fn, window] (or [fn, hop]) on the GPU
            consume(frame)
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .api import BatchPlan, _scales_array


class StreamingCWT:
    """Sliding-window transform of a real signal.

    window, hop: window length and advance in samples (0 < hop <= window).
    emit: "window" returns each frame's full [fn, window] coefficients;
    "hop" returns only the newest `hop` columns of the frame.
    out_type: any FCWT_OUT_* type (complex64, 16-bit pairs, power, dB).
    The first frame is produced once `window` samples have arrived. The last
    frame returned by a call is a view of the output buffer that the next
    frame overwrites (copy it to keep it); earlier frames of the same call are
    copies.
    """

    def __init__(self, window: int, hop: int, scales, fb: float = 2.0, threads: int = 1, norm: bool = True,
                 device: int = 0, out_type: int = _lib.FCWT_OUT_C64, emit: str = "window", graph: bool = True):
        import torch

        if not (0 < hop <= window):
            raise ValueError("need 0 < hop <= window")
        if emit not in ("window", "hop"):
            raise ValueError("emit must be 'window' or 'hop'")
        self.window, self.hop, self.emit, self.graph = int(window), int(hop), emit, bool(graph)
        self.out_type = int(out_type)
        self.scales = _scales_array(scales).copy()
        self.fn = self.scales.size
        self.device = device
        dev = f"cuda:{device}"
        self.plan = BatchPlan([self.window], [self.scales], fb=fb, threads=threads, norm=norm, device=device)
        self.buf = torch.zeros(self.window, dtype=torch.float32, device=dev)
        if self.out_type == _lib.FCWT_OUT_C64:
            self.out = torch.empty((self.fn, self.window), dtype=torch.complex64, device=dev)
        elif self.out_type in (_lib.FCWT_OUT_BF16, _lib.FCWT_OUT_F16):
            dt = torch.bfloat16 if self.out_type == _lib.FCWT_OUT_BF16 else torch.float16
            self.out = torch.empty((self.fn, self.window, 2), dtype=dt, device=dev)
        else:
            self.out = torch.empty((self.fn, self.window), dtype=torch.float32, device=dev)
        self.filled = 0          # samples in the buffer (up to window)
        self.pending = 0         # new samples since the last frame
        self.frames = 0

    def _run(self):
        self.plan.execute([self.buf], [self.out], out_type=self.out_type, graph=self.graph)
        self.frames += 1
        return self.out if self.emit == "window" else self.out[:, self.window - self.hop:]

    def push(self, samples) -> list:
        """Append samples (1-D numpy array or torch tensor); returns the frames
        completed by them, oldest first."""
        import torch

        x = samples if isinstance(samples, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(samples))
        x = x.to(device=self.buf.device, dtype=torch.float32).reshape(-1)
        frames = []
        i = 0
        while i < x.numel():
            if self.filled < self.window:
                take = min(self.window - self.filled, x.numel() - i)
                self.buf[self.filled:self.filled + take] = x[i:i + take]
                self.filled += take
                i += take
                if self.filled == self.window:
                    f = self._run()
                    frames.append(f.clone() if x.numel() - i >= self.hop else f)
                    self.pending = 0
                continue
            take = min(self.hop - self.pending, x.numel() - i)
            # shift the window left by `take` samples and append them
            self.buf[:self.window - take] = self.buf[take:].clone()
            self.buf[self.window - take:] = x[i:i + take]
            self.pending += take
            i += take
            if self.pending == self.hop:
                f = self._run()
                # a later frame of this call overwrites the output buffer: keep a copy
                frames.append(f.clone() if x.numel() - i >= self.hop else f)
                self.pending = 0
        return frames

    def close(self) -> None:
        self.plan.close()
