import torch


def to_dlpack_safe(t: torch.Tensor, stream_ptr: int):
    """del_splat_dlpack/util_torch.py:3-13.  On CUDA, stream handle 0 (what
    ``torch.cuda.current_stream().cuda_stream`` returns for the default
    stream) is passed as 1, the DLPack name of the legacy default stream
    (DLPack disallows 0; torch rejects it)."""
    assert not t.requires_grad
    assert t.is_contiguous()
    dev = t.device.type
    if dev == "cuda":
        return t.__dlpack__(stream=stream_ptr if stream_ptr else 1)
    elif dev == "cpu":
        return t.__dlpack__()
    else:
        raise RuntimeError(f"Unsupported device for DLPack export: {t.device}")
