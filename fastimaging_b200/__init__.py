"""B200-native snapshot imager and source finder (FastImaging hot path).

Public surface:
  fastimaging_b200.capi        ctypes binding of the C ABI (include/stpgpu.h)
  fastimaging_b200.stp_python  drop-in for the reference's pybind11 module
                               (image_visibilities_wrapper, source_find_wrapper,
                               enums, Gaussian2dParams), built by
                               ``python -m fastimaging_b200.build``
"""
__all__ = ["capi", "synthetic"]
