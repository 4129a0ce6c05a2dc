import torch

from .. import _CapsuleAsDLPack


def load_ply(path_file: str):
    """del_splat_dlpack/Points/torch.py:5-12 -> (pnt2xyz [N,3], pnt2rgb [N,3]) CPU tensors."""
    from .. import Points

    cap_pnt2xyz, cap_pnt2rgb = Points.load_ply(path_file)
    pnt2xyz = torch.from_dlpack(_CapsuleAsDLPack(cap_pnt2xyz))
    pnt2rgb = torch.from_dlpack(_CapsuleAsDLPack(cap_pnt2rgb))
    return pnt2xyz, pnt2rgb
