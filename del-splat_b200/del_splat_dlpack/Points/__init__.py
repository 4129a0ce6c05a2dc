def load_ply(path_file: str):
    """del_splat_dlpack/Points/__init__.py:1-4."""
    from ..del_splat_dlpack import points_load_ply

    return points_load_ply(path_file)
