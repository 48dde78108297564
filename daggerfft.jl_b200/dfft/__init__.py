"""dfft: B200-native transform hot path of DaggerFFT.jl (Python host side).

``import dfft`` after putting ``daggerfft.jl_b200`` on ``sys.path``.  The
compute runs in ``libdfft.so`` (hand-written sm_100a CUDA kernels behind a C
ABI, see include/dfft.h); this package is the ctypes host layer that mirrors
the reference's Julia API.
"""
from ._lib import (FLAG_DESTROY_INPUT, FLAG_FUSE, FLAG_NO_FUSE, FLAG_NO_WISDOM, FLAG_TUNE, ArgumentError, DFFTError, LIB_PATH,
                   device_error, lib, wisdom_export, wisdom_forget, wisdom_import, wisdom_size)
from .api import (Batch, DHT, FFT, FFT_, GPU_PLAN_CACHE, HC2R, IFFT, IFFT_, IRFFT, IRFFT_, R2HC, R2R,
                  R2R_SUPPORTED_KINDS, REDFT00, REDFT01, REDFT10, REDFT11, RFFT, RFFT_, RODFT00,
                  RODFT01, RODFT10, RODFT11, Decomposition, Pencil, Plan, Slab, Transform,
                  apply_gpu_fft_, empty_like_layout, fft, fft_, get_or_create_gpu_plan,
                  gpu_cleanup_plans, gpu_plan_transform, ifft, ifft_, irfft, rfft)

from .darray import (Blocks, CudaCopier, DArray, Workspace, collect, compute_overlap,
                     create_gpu_workspace, distribute, empty_darray, gpu_cleanup_workspace_,
                     gpu_coalesced_redistribute_, gpu_fft_, gpu_ifft_)

from .serve import Server
from .slab_dist import FusedSlabFFT, SlabSplitPlan

__version__ = "0.1.0"
