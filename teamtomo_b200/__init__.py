"""teamtomo_b200 — B200-native Fourier-slice path of TeamTomo.

Drop-in replacements for the 3D Fourier-slice API of torch-fourier-slice and
the 3D interpolation API of torch-image-interpolation, running on
hand-written sm_100a CUDA kernels through the C ABI in include/teamtomo_b200.h.
"""

from . import (
    autotune,
    batched,
    distributed,
    losses,
    streaming,
    torch_fourier_slice,
    torch_image_interpolation,
    torch_transform_image,
)
from .torch_fourier_slice import (
    backproject_2d_to_3d,
    backproject_2d_to_3d_multichannel,
    extract_central_slices_rfft_2d,
    extract_central_slices_rfft_3d,
    extract_central_slices_rfft_3d_multichannel,
    insert_central_slices_rfft_3d,
    insert_central_slices_rfft_3d_multichannel,
    project_2d_to_1d,
    project_3d_to_2d,
    project_3d_to_2d_multichannel,
)
from .torch_image_interpolation import insert_into_image_3d, sample_image_3d

__version__ = "0.1.0"

__all__ = [
    "autotune",
    "batched",
    "distributed",
    "losses",
    "streaming",
    "torch_fourier_slice",
    "torch_image_interpolation",
    "torch_transform_image",
    "backproject_2d_to_3d",
    "backproject_2d_to_3d_multichannel",
    "extract_central_slices_rfft_2d",
    "extract_central_slices_rfft_3d",
    "extract_central_slices_rfft_3d_multichannel",
    "insert_central_slices_rfft_3d",
    "insert_central_slices_rfft_3d_multichannel",
    "project_2d_to_1d",
    "project_3d_to_2d",
    "project_3d_to_2d_multichannel",
    "sample_image_3d",
    "insert_into_image_3d",
]
