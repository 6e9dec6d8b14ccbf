"""tom_b200: B200-native (sm_100a) template matching for the TOM toolbox.

The compute lives in libtomgpu.so (tom_b200/csrc, C ABI in include/tomgpu.h),
loaded through ctypes.  The functions below mirror the TOM toolbox's MATLAB
functions on the template-matching path (rotate -> wedge -> FFT correlation ->
FLCF normalisation -> running max/arg-max).
"""
from ._lib import TomGpuError, declared_symbols, lib  # noqa: F401
from .tom import (  # noqa: F401
    Context,
    MatchPlan,
    av3_align_batch,
    av3_align_host,
    av3_average_add,
    av3_average_final,
    av3_tomomatch_average,
    av3_wedge,
    default_context,
    euler_matrix,
    from_device,
    match_host,
    pick_peaks,
    picklist_to_motl,
    to_device,
    tom_av3_align,
    tom_av3_angle2index,
    tom_av3_angle_grid,
    tom_av3_index2angle,
    tom_apply_weight_function,
    tom_calc_weight_functioninc,
    cpp_spheremask,
    tom_corr,
    tom_corr3d,
    tom_emread,
    tom_emwrite,
    tom_fourier,
    tom_ifourier,
    tom_os3_analyzePeak,
    tom_os3_angleList,
    tom_os3_corr,
    tom_os3_findTemplate,
    tom_os3_sphereMask,
    tom_os3_template_autocorr,
    tom_peak,
    tom_peakc,
    tom_rotate,
    tom_rotatec,
    tom_wedge,
    topk_peaks,
)

__version__ = "0.1.0"
