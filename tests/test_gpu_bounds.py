"""The bounds-checked debug build (libfsl_gpu_checked.so): every step path
whose kernels carry the checks (FP64 and FP32 ring tiles, the FP32 full-lane
tile, the per-phase kernels, PPM, the dynamic procedure in both precisions,
the static and learned closures, the persistent ensemble, the Courant and
conservation reductions, probes and Tecplot fields, the state scatter/gather
of the asynchronous transfers, the allocation-free SGS entry point), on grids
with partial tiles in every direction and on both setups, makes no
out-of-range global-memory access.  The workload runs in a child process
that loads the checked library (FSL_GPU_LIB=checked); this file is also that
child."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _workload():
    sys.path.insert(0, ROOT)
    import freeshearlayer_b200 as fsl
    from tests.helpers import spatial_params, temporal_params

    assert fsl.LIB_PATH.endswith("libfsl_gpu_checked.so"), fsl.LIB_PATH
    fsl.debug_bounds(clear=True)
    runs = 0

    def temporal(L, H, D, **kw):
        p = temporal_params(L=L, H=H, D=D, Mc=0.5, **kw)
        s, dU = fsl.temporal_state(p, 0.5, 1.0, 2e-2, L + H + D)
        d = fsl.Domain(p)
        d.upload_state(s)
        if kw.get("sgs") == 1:
            d.closure_set_scales(1.0 / dU, 1.0)
            d.closure_set_weights(fsl.closure_weights())
            d.closure_judge(0, 1.0)
        return d, s

    # spatial setup (the reference's boundary rules, disturbance block),
    # both precisions, fused and per-phase
    for prec in (0, 1):
        d = fsl.Domain(spatial_params(L=13, H=10, D=7, precision=prec))
        d.upload_state(fsl.initial_state(spatial_params(L=13, H=10, D=7)))
        d.step(3)
        if prec == 0:
            d.step_phased(1)
        assert np.all(np.isfinite(d.download_state()))
        runs += 1
    # per-phase kernels (PPM too), the Courant and conservation reductions,
    # probes, Favre sums and Tecplot fields, on both setups
    for p in (spatial_params(L=13, H=10, D=7), temporal_params(L=15, H=11, D=9, recon=1)):
        d = fsl.Domain(p)
        d.upload_state(fsl.initial_state(p) if p["setup"] == 0 else fsl.temporal_state(p, 0.4, 1.0, 2e-2, 3)[0])
        d.step_phased(2)
        d.check_courant()
        d.sums()
        d.plane_sums()
        d.probe_rows()
        d.favre_reset()
        d.favre_accumulate()
        assert np.all(np.isfinite(d.output_fields()))
        runs += 1
    # temporal setup: partial tiles in y and z (full lane 16 x 32, ring
    # tiles of 8, 12, 16 rows), odd extents; static and no SGS; PPM
    for prec in (0, 1):
        for rows in ((0, 8, 12, 16) if prec == 1 else (8, 12, 16)):
            for sgs in (0, 2, 3):
                d, _ = temporal(19, 21, 35, precision=prec, sgs=sgs)
                d.tune(d.TUNE_STAGE_ROWS, rows)
                d.step(2)
                runs += 1
        d, _ = temporal(17, 13, 33, precision=prec, recon=1)
        d.step(2)
        runs += 1
    # learned closure (inference on the stage-written velocities, a
    # judgement with the dynamic procedure beside it), long x march
    d, s = temporal(70, 18, 34, precision=1, sgs=1)
    d.step(3)
    # asynchronous transfers: state scatter and gather
    out = np.empty_like(s)
    d.upload_state_async(s)
    d.step(1)
    d.download_state_async(out)
    d.transfer_wait()
    assert np.all(np.isfinite(out))
    runs += 1
    # persistent ensemble of uneven members
    members = [temporal(24, 16, 16, precision=1)[0], temporal(20, 12, 36, precision=1, sgs=1)[0],
               temporal(16, 20, 12, precision=1)[0]]
    e = fsl.Ensemble(members)
    e.step(4)
    e.sync()
    e.close()
    runs += 1
    # the allocation-free SGS entry point (the unfused dynamic procedure on
    # its static scratch array), on a padded state with its ghost layer
    import ctypes as C

    import torch
    p = temporal_params(L=19, H=13, D=17, Mc=0.5)
    s, _ = fsl.temporal_state(p, 0.5, 1.0, 2e-2, 11)
    d = fsl.Domain(p)
    d.upload_state(s)
    d.ghost_bc()
    U = torch.from_numpy(np.ascontiguousarray(np.stack([d.cells(0, v) for v in range(4)]))).cuda()
    mu = torch.zeros(d.cells(3).shape, dtype=torch.float64, device="cuda")
    fn = fsl.lib().fsl_dynamic_smagorinsky_noalloc
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                   C.c_void_p]
    fn.restype = C.c_int
    torch.cuda.synchronize()
    rc = fn(U.data_ptr(), mu.data_ptr(), p["LEN"], p["HIG"], p["DEP"], p["deltaX"], p["deltaY"], p["deltaZ"],
            C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, rc
    torch.cuda.synchronize()
    runs += 1
    rep = fsl.debug_bounds()
    rep["runs"] = runs
    print(json.dumps(rep))


@pytest.mark.gpu
def test_checked_build_finds_no_out_of_range_access():
    lib = os.path.join(ROOT, "freeshearlayer_b200", "libfsl_gpu_checked.so")
    assert os.path.exists(lib), "build it: make -C freeshearlayer_b200 checked"
    env = dict(os.environ, FSL_GPU_LIB="checked")
    r = subprocess.run([sys.executable, os.path.abspath(__file__)], env=env, cwd=ROOT, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    rep = json.loads(r.stdout.strip().splitlines()[-1])
    assert rep["runs"] >= 28
    assert rep["hits"] == 0, rep


def test_product_build_has_no_checks():
    """The product library reports FSL_ERR_UNSUPPORTED (no device work)."""
    import freeshearlayer_b200 as fsl
    if not fsl.LIB_PATH.endswith("libfsl_gpu.so"):
        pytest.skip("FSL_GPU_LIB selects another build")
    with pytest.raises(fsl.FslError) as ex:
        fsl.debug_bounds()
    assert ex.value.code == -7
    assert fsl.lib().fsl_debug_bounds(None, 0) == -1  # no report to fill: FSL_ERR_ARG


if __name__ == "__main__":
    _workload()
