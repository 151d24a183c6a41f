"""gemsgpu_smatb_forces_noalloc against the context entry point (GPU).

The no-allocation entry point serves callers that cannot allocate device
memory -- a host that gives the library only buffers from its own fixed
device budget, or code evaluating forces where cudaMalloc/cudaFree are not
allowed (they synchronise the device and are refused during CUDA-graph
capture).  Its forces and energies must equal those of gemsgpu_forces (the
list-based FP64 SMA-TB path) within the FP64 tolerances of the other GPU
tests, on two calls in a row (the second reuses the shared scratch array).
This file sorts last so a stop-at-first-failure run reaches it only after
every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RMS_FP64 = 1e-10   # relative RMS of forces, as in test_gpu_parity
E_FP64 = 1e-9      # eV per atom


def test_noalloc_matches_context_entry_point():
    torch = pytest.importorskip("torch")
    import gems_b200 as gems
    from gems_b200 import workloads as W

    w = W.smatb_bulk(ncell=8)               # 2048 Au atoms, periodic
    n = len(w["pos"])
    ctx = gems.Context()
    try:
        g = gems.System(w["pos"], w["mass"], ctx=ctx)
        g.set_box(w["L"], (True, True, True))
        g.set_smatb(*w["smatb"])
        g.interact()
        f_ref, e_ref = g.force, g.epot_atoms
    finally:
        ctx.close()

    fn = gems.lib().gemsgpu_smatb_forces_noalloc
    dev = torch.device("cuda", 0)
    d_pos = torch.tensor(w["pos"].ravel(), dtype=torch.float64, device=dev)
    d_force = torch.empty(3 * n, dtype=torch.float64, device=dev)
    d_epot = torch.empty(n, dtype=torch.float64, device=dev)
    L = np.ascontiguousarray(w["L"], dtype=np.float64)
    pbc = np.ones(3, dtype=np.int32)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)

    def call(nat):
        return fn(ctypes.c_void_p(d_pos.data_ptr()), nat, 1,
                  L.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                  pbc.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                  *w["smatb"], ctypes.c_void_p(d_force.data_ptr()),
                  ctypes.c_void_p(d_epot.data_ptr()), stream)

    for _ in range(2):
        d_force.fill_(float("nan"))
        d_epot.fill_(float("nan"))
        assert call(n) == 0
        torch.cuda.synchronize()
        f = d_force.cpu().numpy().reshape(n, 3)
        e = d_epot.cpu().numpy()
        rms = np.linalg.norm(f - f_ref) / np.linalg.norm(f_ref)
        assert rms <= RMS_FP64, rms
        assert np.abs(e - e_ref).max() * gems.UI_EV <= E_FP64

    # sizes beyond the fixed scratch are refused before any launch
    assert call(16385) == -10     # GEMSGPU_ERR_FULL


def test_noalloc_open_cluster_matches_oracle():
    """boxed = 0: a free 600-atom Au cluster (no periodic dimension), two
    calls in a row, against the FP64 oracle's smatb_interact directly."""
    torch = pytest.importorskip("torch")
    import gems_b200 as gems
    from gems_b200 import workloads as W
    from oracle import oracle as O

    pos = W.cluster(600, np.random.default_rng(12))
    n = len(pos)
    o = O.System(pos, W.MASS["Au"])
    o.set_smatb(*W.SMATB["Au"])
    o.interact()
    f_ref, e_ref = o.force, o.epot_atoms

    fn = gems.lib().gemsgpu_smatb_forces_noalloc
    dev = torch.device("cuda", 0)
    d_pos = torch.tensor(pos.ravel(), dtype=torch.float64, device=dev)
    d_force = torch.empty(3 * n, dtype=torch.float64, device=dev)
    d_epot = torch.empty(n, dtype=torch.float64, device=dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    for _ in range(2):
        d_force.fill_(float("nan"))
        d_epot.fill_(float("nan"))
        rc = fn(ctypes.c_void_p(d_pos.data_ptr()), n, 0, None, None, *W.SMATB["Au"],
                ctypes.c_void_p(d_force.data_ptr()), ctypes.c_void_p(d_epot.data_ptr()), stream)
        assert rc == 0
        torch.cuda.synchronize()
        f = d_force.cpu().numpy().reshape(n, 3)
        e = d_epot.cpu().numpy()
        rms = np.linalg.norm(f - f_ref) / np.linalg.norm(f_ref)
        assert rms <= RMS_FP64, rms
        assert np.abs(e - e_ref).max() * gems.UI_EV <= E_FP64
