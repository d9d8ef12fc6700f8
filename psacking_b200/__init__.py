"""psacking_b200 — B200-native placement search for spectral 3D packing.

A drop-in for the hot path of Vrroom/psacking: the module `_core` exposes the
reference's `spectral_packer._core` functions (spectral_packing/bindings.cpp:
654-930) on hand-written sm_100a kernels behind the C ABI in include/psb200.h;
`BinPacker` mirrors spectral_packer.packer.BinPacker.

The extension is required: importing this package without the built
libpsb200.so / _core module raises ImportError (run python psacking_b200/build.py).
"""
from __future__ import annotations

try:
    from . import _core
except ImportError as e:  # fail loudly: there is no CPU fallback
    raise ImportError(
        "psacking_b200._core is not built (python psacking_b200/build.py): " + str(e)) from e

from ._core import (  # noqa: E402
    HEIGHT_PENALTY,
    VOXEL_RESOLUTION,
    calculate_distance,
    collision_grid,
    dft_conv3,
    dft_corr3,
    fft_search_batch,
    fft_search_batch_interlocking_free,
    fft_search_placement,
    fft_search_placement_with_cache,
    get_bounds,
    gpu_tray_cleanup,
    gpu_tray_init,
    gpu_tray_is_initialized,
    gpu_tray_search,
    interlocking_free_positions,
    make_tight,
    place_in_tray,
)
from .packer import BinPacker, PackingResult, PlacementInfo  # noqa: E402
from .rotations import (  # noqa: E402
    ROTATION_MATRICES_3x3,
    get_24_orientations,
    get_orientations,
    get_rotation_matrix_3x3,
    get_rotation_matrix_4x4,
    orientation_maps,
    rotate_90_x,
    rotate_90_y,
    rotate_90_z,
)
from .vox import save_vox  # noqa: E402

__version__ = _core.__version__


def is_cuda_available() -> bool:
    """spectral_packer.is_cuda_available (__init__.py:163-172 of the
    reference), which is always True there because its module imports only
    with CUDA support.  Here the extension also imports on a machine without
    a GPU (its calls then raise), so this reports whether a CUDA device is
    visible to the engine."""
    return _core.device_count() > 0


def voxelize_stl(path, resolution: int = VOXEL_RESOLUTION):
    """The reference's mesh voxelizer (bindings.cpp:285-302): surface voxels
    of a binary or ASCII STL mesh, tight int32 grid (psacking_b200.voxelize)."""
    from .voxelize import voxelize_stl as _v
    return _v(path, resolution)


__all__ = [
    "__version__", "is_cuda_available", "BinPacker", "PackingResult", "PlacementInfo", "HEIGHT_PENALTY", "VOXEL_RESOLUTION",
    "calculate_distance", "collision_grid", "dft_conv3", "dft_corr3", "fft_search_batch",
    "fft_search_batch_interlocking_free", "fft_search_placement", "fft_search_placement_with_cache",
    "get_bounds", "gpu_tray_cleanup", "gpu_tray_init", "gpu_tray_is_initialized", "gpu_tray_search",
    "interlocking_free_positions", "make_tight", "place_in_tray", "save_vox", "voxelize_stl",
    "get_orientations", "get_24_orientations", "orientation_maps", "rotate_90_x", "rotate_90_y",
    "rotate_90_z", "get_rotation_matrix_3x3", "get_rotation_matrix_4x4", "ROTATION_MATRICES_3x3",
]
