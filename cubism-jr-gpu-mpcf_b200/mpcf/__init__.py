"""mpcf: host layer of libmpcf_b200, the B200 implementation of the
CUBISM-MPCF per-step hot path (WENO5/HLLC convection, LSRK3 stage update,
maximum speed of sound)."""
from ._lib import (BC_ABSORBING, BC_REFLECTING, BC_HALO, PREC_FP32_REF, PREC_FP32, PREC_MIXED, PREC_FP64,
                   PRECISIONS, MpcfError, IcParams, SicParams, lib, LIB_PATH)
from .solver import (Solver, WindowSolver, window_plan, window_stage_plan, GPUlab, lsrk3_step, ic_cloud_host, bubbles, LSRK3, FIELDS,
                     dtype_of, sic_params, sic_post_shock, case_params, case_bc)
from . import configs

__all__ = ["BC_ABSORBING", "BC_REFLECTING", "BC_HALO", "PREC_FP32_REF", "PREC_FP32", "PREC_MIXED", "PREC_FP64",
           "PRECISIONS", "MpcfError", "IcParams", "SicParams", "lib", "LIB_PATH", "Solver", "WindowSolver", "window_plan", "window_stage_plan",
           "GPUlab", "lsrk3_step",
           "ic_cloud_host", "bubbles", "LSRK3", "FIELDS", "dtype_of", "configs", "sic_params", "sic_post_shock", "case_params", "case_bc"]
