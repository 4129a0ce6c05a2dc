"""del_splat_dlpack -- drop-in replacement of del-splat's Python package.

Same package layout and function names as del-splat-dlpack
(del_splat_dlpack/{SplatCircle,SplatPoint,Points}/{__init__,torch}.py and the
extension functions of del-splat-dlpack/src/lib.rs:9-15), backed by
libdsplat.so.  The GPU branch is the only compute path: CPU tensors raise
(the reference dispatched them to del-splat-cpu).  Added: SplatGauss, the
Gaussian projection / tile lists / raster and a differentiable batched render.
"""


class _CapsuleAsDLPack:
    """del_splat_dlpack/__init__.py:1-14 -- wraps a DLPack capsule for torch.from_dlpack."""

    def __init__(self, cap):
        self._cap = cap
        self._used = False

    def __dlpack__(self, *, max_version=None, stream=None):
        if self._used:
            raise RuntimeError("DLPack capsule already consumed")
        self._used = True
        return self._cap

    def __dlpack_device__(self):
        return (1, 0)
