"""Fourier slice extraction / insertion on B200 (drop-in for torch_fourier_slice).

Same public names, signatures, defaults, return types and exceptions as
torch_fourier_slice/__init__.py:16-42: the 3D path and the 2D central lines.
"""

from .backproject import backproject_2d_to_3d, backproject_2d_to_3d_multichannel
from .lines_2d import extract_central_slices_rfft_2d, project_2d_to_1d
from .project import project_3d_to_2d, project_3d_to_2d_multichannel
from .slice_extraction import (
    extract_central_slices_rfft_3d,
    extract_central_slices_rfft_3d_multichannel,
)
from .slice_insertion import (
    insert_central_slices_rfft_3d,
    insert_central_slices_rfft_3d_multichannel,
)

__all__ = [
    "backproject_2d_to_3d",
    "backproject_2d_to_3d_multichannel",
    "project_3d_to_2d",
    "project_3d_to_2d_multichannel",
    "project_2d_to_1d",
    "extract_central_slices_rfft_3d",
    "extract_central_slices_rfft_3d_multichannel",
    "extract_central_slices_rfft_2d",
    "insert_central_slices_rfft_3d",
    "insert_central_slices_rfft_3d_multichannel",
]
