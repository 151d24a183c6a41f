"""B200 (sm_100a) force/neighbour path of the GEMS molecular simulator.

The compute lives in libgemsgpu.so (hand-written CUDA behind the C ABI of
include/gemsgpu.h); this package is the thin host-side binding.
"""
from .gemsgpu import (Context, GemsGpuError, System, Pool, Server,  # noqa: F401
                      PREC_FP64, PREC_MIXED, FF_LJ, FF_SMATB, FF_TERSOFF,
                      JOB_FIRE, JOB_MD, JOB_QUEUED, JOB_RUNNING, JOB_DONE, JOB_FAILED,
                      UI_EV, EV_UI, KB_UI, lib, declared_symbols, measure_peaks)
