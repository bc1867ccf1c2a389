"""rtfmm_b200: the periodic kernel-independent Laplace FMM evaluation pass of
mumairsadiq/exafmm-rd (variant 3dpp), rebuilt for NVIDIA B200 (sm_100a).

The compute path is librtfmm_b200.so (C ABI in include/rtfmm_b200.h); this
package is its Python mirror of the reference driver interface.  The
directory name is not a Python identifier, so load it by path:

    import importlib.util, os
    spec = importlib.util.spec_from_file_location(
        "exafmm_rd_b200", os.path.join(root, "exafmm-rd_b200", "__init__.py"),
        submodule_search_locations=[os.path.join(root, "exafmm-rd_b200")])
    pkg = importlib.util.module_from_spec(spec); spec.loader.exec_module(pkg)
"""
from .rtfmm import (FP32_MIXED, FP64, STAGE_ALL, STAGE_FAR, STAGE_NAMES, STAGE_NEAR, STAGE_SERIAL, STAGE_TIMED,
                    Argument, LaplaceFMM, RtfmmError, clear_operator_cache, load_operators, compare, direct_sampled, ewald_sampled, generate_random_bodies, lib)

__all__ = ["Argument", "LaplaceFMM", "RtfmmError", "clear_operator_cache", "load_operators", "compare", "direct_sampled", "ewald_sampled",
           "generate_random_bodies", "lib", "FP64",
           "FP32_MIXED", "STAGE_ALL", "STAGE_FAR", "STAGE_NEAR", "STAGE_NAMES", "STAGE_SERIAL", "STAGE_TIMED"]
