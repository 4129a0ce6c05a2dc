"""dsplat.feed.HostToDeviceFeed: each step sees exactly its own inputs while
the next step's copy overlaps it, slots are reused only after their step, and
misuse raises."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_feed_delivers_each_steps_inputs_in_order(dev):
    from dsplat.feed import HostToDeviceFeed
    n = 1 << 22  # 16 MB per tensor: copies long enough to overlap the consumer
    steps = [{"a": torch.full((n,), float(k)).pin_memory(), "b": torch.arange(8, dtype=torch.int32).pin_memory() + k}
             for k in range(5)]
    feed = HostToDeviceFeed(steps[0], dev)
    seen = []
    feed.put(steps[0])
    for k in range(5):
        d = feed.get()
        if k + 1 < 5:
            feed.put(steps[k + 1])
        # a consumer that takes a while and reads the whole slot
        acc = torch.zeros((), device=dev)
        for _ in range(8):
            acc = acc + d["a"].sum()
        seen.append((acc / (8 * n), d["b"].clone()))
        feed.release()
    torch.cuda.synchronize(dev)
    for k, (mean, b) in enumerate(seen):
        assert float(mean) == float(k)
        assert np.array_equal(b.cpu().numpy(), np.arange(8) + k)


def test_feed_rejects_misuse(dev):
    from dsplat.feed import HostToDeviceFeed
    host = {"a": torch.zeros(4).pin_memory()}
    feed = HostToDeviceFeed(host, dev, slots=2)
    with pytest.raises(RuntimeError):
        feed.get()
    with pytest.raises(RuntimeError):
        feed.release()
    feed.put(host)
    feed.put(host)
    with pytest.raises(RuntimeError):
        feed.put(host)  # both slots hold inputs nobody took
