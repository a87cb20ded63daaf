"""B200-native 2D kernel-independent FMM with the interface of dbstein/pykifmm2d.

    from pykifmm2d_b200 import FMM, Get_Kernel_Functions, \
        prepare_numba_functions_on_the_fly, LaplaceKernel
    kern = LaplaceKernel()
    fmm = FMM(x, y, Get_Kernel_Functions(kern), prepare_numba_functions_on_the_fly(kern),
              Nequiv=32, Ncutoff=64)
    fmm.build_tree(); fmm.precompute(); fmm.build_expansions(tau)
    pot = fmm.evaluate_to_points(x, y, check_self=True)

The work runs in libkifmm2d.so (hand-written sm_100a CUDA, C ABI in
include/kifmm2d.h); this package is the Python host layer.
"""
from . import class_fmm
from .class_fmm import (FMM, Get_Kernel_Functions, HelmholtzKernel, Kernel_Form, LaplaceKernel,
                        ModifiedHelmholtzKernel, get_level_information, prepare_numba_functions_on_the_fly)

__all__ = ["FMM", "Get_Kernel_Functions", "Kernel_Form", "LaplaceKernel", "ModifiedHelmholtzKernel",
           "HelmholtzKernel", "get_level_information", "prepare_numba_functions_on_the_fly", "class_fmm"]
