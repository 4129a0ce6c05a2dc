"""Double-buffered host -> device input feed for training / rendering loops.

A step's inputs (parameters streamed from the host, target images, ...) are
copied from pinned host memory into one of two device slots on a side CUDA
stream, so the copy for step k+1 runs while step k computes.  The compute
stream waits for a slot's copy before using it, and the copy into a slot
waits until the step that last used it has finished, so no slot is
overwritten while a kernel still reads it.

    feed = HostToDeviceFeed({"means": host_means, "target": host_target}, device)
    feed.put(host_inputs_0)
    for k in range(steps):
        dev = feed.get()              # current stream waits for the copy
        if k + 1 < steps:
            feed.put(host_inputs[k + 1])   # overlaps with the step below
        run_step(dev)
        feed.release()                # the slot may be refilled after this point

Host tensors passed to put() must be pinned (page-locked) for the copies to
be asynchronous.
"""
from __future__ import annotations

from typing import Dict, Optional

import torch


class HostToDeviceFeed:
    def __init__(self, like: Dict[str, torch.Tensor], device: torch.device, slots: int = 2):
        if slots < 1:
            raise ValueError("slots must be >= 1")
        self.device = torch.device(device)
        self.copy_stream = torch.cuda.Stream(device=self.device)
        self.slots = [{k: torch.empty(v.shape, dtype=v.dtype, device=self.device) for k, v in like.items()}
                      for _ in range(slots)]
        self.ready = [torch.cuda.Event() for _ in range(slots)]
        self.free = [torch.cuda.Event() for _ in range(slots)]
        self.used = [False] * slots
        self.n_put = 0
        self.n_get = 0
        self.current: Optional[int] = None

    def put(self, host: Dict[str, torch.Tensor]) -> None:
        """Queue the copy of one step's inputs into the next slot."""
        if self.n_put - self.n_get >= len(self.slots):
            raise RuntimeError("all slots hold inputs that were not taken with get()")
        i = self.n_put % len(self.slots)
        with torch.cuda.stream(self.copy_stream):
            if self.used[i]:
                self.copy_stream.wait_event(self.free[i])
            for k, dst in self.slots[i].items():
                dst.copy_(host[k], non_blocking=True)
            self.ready[i].record(self.copy_stream)
        self.n_put += 1

    def get(self) -> Dict[str, torch.Tensor]:
        """Device tensors of the oldest queued step; the current stream waits
        for their copy."""
        if self.n_get >= self.n_put:
            raise RuntimeError("get() without a matching put()")
        i = self.n_get % len(self.slots)
        torch.cuda.current_stream(self.device).wait_event(self.ready[i])
        self.current = i
        self.n_get += 1
        return self.slots[i]

    def release(self) -> None:
        """Mark the slot returned by the last get() as reusable once the work
        queued so far on the current stream has finished."""
        if self.current is None:
            raise RuntimeError("release() without get()")
        self.free[self.current].record(torch.cuda.current_stream(self.device))
        self.used[self.current] = True
        self.current = None


class DeviceToHostDrain:
    """Double-buffered device -> host readback of a step's results.

    push(i, tensors) queues, on a side stream, the copy of device tensors
    written by the work queued so far on the current stream into host slot i
    (pinned), so the copy of step k's results runs while step k+1 computes.
    Before the current stream overwrites those device tensors again it calls
    reclaim(i), which makes it wait for that copy; wait(i) blocks the host
    until slot i's copy has landed and returns its host tensors.

        drain = DeviceToHostDrain({"image": dev_image}, device)
        for k in range(steps):
            drain.reclaim(k % 2)
            render_into(out[k % 2])
            drain.push(k % 2, {"image": out[k % 2]})
        drain.wait((steps - 1) % 2)
    """

    def __init__(self, like: Dict[str, torch.Tensor], device: torch.device, slots: int = 2):
        if slots < 1:
            raise ValueError("slots must be >= 1")
        self.device = torch.device(device)
        self.copy_stream = torch.cuda.Stream(device=self.device)
        self.host = [{k: torch.empty(v.shape, dtype=v.dtype).pin_memory() for k, v in like.items()}
                     for _ in range(slots)]
        self.done = [torch.cuda.Event() for _ in range(slots)]
        self.pending = [False] * slots

    def bytes_per_push(self) -> int:
        return sum(t.numel() * t.element_size() for t in self.host[0].values())

    def reclaim(self, i: int) -> None:
        """The current stream waits until slot i's last copy has read its
        device tensors."""
        if self.pending[i]:
            torch.cuda.current_stream(self.device).wait_event(self.done[i])

    def push(self, i: int, dev: Dict[str, torch.Tensor]) -> None:
        produced = torch.cuda.Event()
        produced.record(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(self.copy_stream):
            self.copy_stream.wait_event(produced)
            for k, dst in self.host[i].items():
                dst.copy_(dev[k], non_blocking=True)
            self.done[i].record(self.copy_stream)
        self.pending[i] = True

    def wait(self, i: int) -> Dict[str, torch.Tensor]:
        if self.pending[i]:
            self.done[i].synchronize()
        return self.host[i]
