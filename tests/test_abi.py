"""C ABI and host logic without a GPU: the library loads, exports every entry
point include/fsl_gpu.h declares, parses layer2.ini / mpi_layer2.bin the way
the reference does, validates parameters, builds initial states identical to
the oracle's, and refuses to run without an sm_100 device (no CPU path)."""
import ctypes as C
import os
import re
import struct
import subprocess

import numpy as np
import pytest

from tests.helpers import spatial_params, temporal_params

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fsl_gpu.h")

# the reference's shipped layer2.ini (22 positional lines with trailing text)
SHIPPED_INI = """100 120        LEN      Number of cells in length     [-]
80  90         HIG      Number of cells in height     [-]
35  41         DEP      Number of cells in depth      [-]
1.6666667  deltaX   X-step                        [m]
1.         deltaY   Y-step                        [m]
1.5        deltaZ   Z-step                        [m]
0.0007     deltaT   Time step                     [sec]
0         Answer   1-continue, 0-start new	      [boolean]
3000      numstep  Number of overall time steps  [-]
0.253358   mu_L     Dynamic mol. viscosity 	      [Pa*sec]
0.72       Pr_L     Mol. Prandtl number
0.8        Pr_T     Turb. Prandtl number
0.01       Cs       Square of the Smagorinsky constant
5          BL_HIG   Height of the random disturbing block
35.        Ua       Amplitude of disturbed U      [m/sec]
35.        Va       Amplitude of disturbed V	  [m/sec]
35.        Wa       Amplitude of disturbed W	  [m/sec]
10         Nst_min  Minimal period of disturbing block
50         Nst      Its max-min
50         f_step   Frame taking step (!output for winfield.exe!)
2          nStages  number of stages (2,3) of TVD Runge-Kutta Algorithm
0.1        maxCoNum    Maximum Courant number for timestepping stability
"""


@pytest.fixture(scope="module")
def fsl():
    import freeshearlayer_b200 as fsl
    fsl.lib()
    return fsl


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(fsl_[a-z0-9_]+)\s*\(", src)))


def test_header_declarations_exported(fsl):
    names = declared_functions()
    assert len(names) > 30
    lib = C.CDLL(fsl.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_checked_build_exports_the_same_abi(fsl):
    """libfsl_gpu_checked.so (the bounds-checked debug build) is a drop-in
    for libfsl_gpu.so: every declared entry point, the bounds report among
    them.  Loaded on the CPU only; no entry point is called."""
    path = os.path.join(os.path.dirname(fsl.LIB_PATH), "libfsl_gpu_checked.so")
    if not os.path.exists(path):
        pytest.skip("libfsl_gpu_checked.so not built (make -C freeshearlayer_b200 checked)")
    lib = C.CDLL(path)
    names = declared_functions()
    assert "fsl_debug_bounds" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_params_from_ini_matches_reference_parser(fsl, tmp_path):
    path = tmp_path / "layer2.ini"
    path.write_text(SHIPPED_INI)
    p = fsl.params_from_ini(str(path))
    assert (p.LEN, p.HIG, p.DEP) == (100, 80, 35)
    assert p.deltaX == 1.6666667 and p.deltaY == 1.0 and p.deltaZ == 1.5 and p.deltaT == 0.0007
    assert p.numstep == 3000 and p.BL_HIG == 5 and p.Ns_min == 10 and p.Nst == 50
    assert p.nStages == 2 and p.maxCoNum == 0.1 and p.mu_L == 0.253358 and p.Cs == 0.01
    short = tmp_path / "short.ini"
    short.write_text("\n".join(SHIPPED_INI.splitlines()[:10]) + "\n")
    with pytest.raises(fsl.FslError) as e:
        fsl.params_from_ini(str(short))
    assert e.value.code == -6


def test_params_from_bin(fsl, tmp_path):
    vals = [64, 32, 32, 0.1, 0.1, 0.1, 1e-4, 0, 200, 0.6, 0.72, 0.8, 0.01, 4, 35, 35, 35,
            10, 50, 50, 3, 0.5]
    path = tmp_path / "mpi_layer2.bin"
    path.write_bytes(struct.pack("<22f", *vals))
    p = fsl.params_from_bin(str(path))
    assert (p.LEN, p.HIG, p.DEP, p.numstep, p.nStages, p.BL_HIG) == (64, 32, 32, 200, 3, 4)
    assert p.deltaX == float(np.float32(0.1)) and p.maxCoNum == float(np.float32(0.5))


def test_unreadable_inputs_are_errors(fsl, tmp_path):
    """Missing or truncated input files return FSL_ERR_IO; text the reference's
    atoi/atof read as zeros parses like the reference and then fails the
    parameter check (FSL_ERR_ARG) before any device work."""
    for fn in (fsl.params_from_ini, fsl.params_from_bin):
        with pytest.raises(fsl.FslError) as e:
            fn(str(tmp_path / "absent"))
        assert e.value.code == -6
    short = tmp_path / "short.bin"
    short.write_bytes(struct.pack("<10f", *range(10)))
    with pytest.raises(fsl.FslError) as e:
        fsl.params_from_bin(str(short))
    assert e.value.code == -6
    junk = tmp_path / "junk.ini"
    junk.write_text("x\n" * 22)
    p = fsl.params_from_ini(str(junk))
    assert (p.LEN, p.HIG, p.DEP, p.deltaX) == (0, 0, 0, 0.0)
    assert fsl.lib().fsl_params_check(C.byref(p)) == -1


def test_plane_buffers_are_checked(fsl):
    """Buffers handed to the plane and transfer calls: contiguous float64 of
    at least the needed length, numpy or torch, else an error before any
    call into the library."""
    import torch
    ok = np.zeros(12)
    assert fsl._buffer_ptr(ok, 12) == ok.ctypes.data
    assert fsl._buffer_ptr(torch.zeros(12, dtype=torch.float64), 12) != 0
    for bad in (np.zeros(11), np.zeros(12, np.float32), np.zeros((12, 2))[:, 0],
                torch.zeros(12, dtype=torch.float32), [0.0] * 12):
        with pytest.raises(fsl.FslError):
            fsl._buffer_ptr(bad, 12)


def test_params_check(fsl):
    lib = fsl.lib()
    ok = fsl.default_params()
    assert lib.fsl_params_check(C.byref(ok)) == 0
    for bad in [dict(BL_HIG=100), dict(LEN=1), dict(deltaX=0.0), dict(nStages=4), dict(setup=7),
                dict(cfl_mode=3), dict(maxCoNum=-1.0)]:
        p = fsl.default_params(**bad)
        assert lib.fsl_params_check(C.byref(p)) == -1, bad
    # PPM runs on the fused step in both precisions
    assert lib.fsl_params_check(C.byref(fsl.default_params(recon=fsl.RECON_PPM))) == 0
    assert lib.fsl_params_check(C.byref(fsl.default_params(recon=fsl.RECON_PPM, precision=1))) == 0
    assert lib.fsl_params_check(C.byref(fsl.default_params(recon=2))) == -1


def test_shear_statistics_tanh_profile(fsl):
    """theta of u = dU/2 tanh(2y/delta) at uniform density is delta/4."""
    H, nrow, dU, delta = 4000, 6, 3.0, 1.0
    dy = 20.0 / H
    y = (np.arange(H) + 0.5) * dy - 10.0
    u = 0.5 * dU * np.tanh(2 * y / delta)
    rows = np.zeros((H, 8))
    rows[:, 0] = nrow
    rows[:, 1] = nrow * u
    rows[:, 4] = nrow * u * u + nrow * 0.25
    rows[:, 7] = nrow * u * 0.1
    st = fsl.shear_statistics(rows, nrow, dU, dy)
    assert abs(st["theta"] - delta / 4) < 1e-6
    np.testing.assert_allclose(st["R11"], 0.25, atol=1e-12)
    np.testing.assert_allclose(st["R12"], 0.1 * u, atol=1e-12)


def test_initial_states_match_oracle(fsl, oracle_lib):
    p = spatial_params(L=9, H=7, D=5)
    assert np.array_equal(fsl.initial_state(p), oracle_lib.spatial_initial_state(p))
    q = temporal_params(L=12, H=8, D=6)
    a, dUa = fsl.temporal_state(q, 0.4)
    b, dUb = oracle_lib.Oracle.temporal_state(q, 0.4)
    assert dUa == dUb and np.array_equal(a, b)


def test_no_cpu_fallback(fsl):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(fsl.FslError) as e:
        fsl.Domain(spatial_params())
    assert e.value.code == -8


@pytest.mark.parametrize("real_bytes", [4, 8])
def test_favre_post_processor(fsl, tmp_path, real_bytes):
    """favre-average-src/layer2_p.c over a probes file: records inside the
    step window summed per station and row, u~ = sum(rho u) / sum(rho); the
    read stops past step_end and at the end of the file."""
    H = 7
    rng = np.random.default_rng(3)
    dt = np.float32 if real_bytes == 4 else np.float64
    recs = []
    path = tmp_path / "probes.dat"
    with open(path, "wb") as f:
        for step in range(1, 11):
            rho = (1.0 + 0.1 * rng.random((3, H))).astype(dt)
            ru = (100.0 * rng.random((3, H))).astype(dt)
            f.write(np.int32(step).tobytes())
            for s in range(3):
                f.write(rho[s].tobytes())
                f.write(ru[s].tobytes())
            recs.append((step, rho.astype(np.float64), ru.astype(np.float64)))
    u, n = fsl.favre_from_probes(str(path), H, real_bytes, 3, 8)
    sel = [r for r in recs if 3 <= r[0] <= 8]
    R = sum(r[1] for r in sel)
    RU = sum(r[2] for r in sel)
    assert n == 6
    np.testing.assert_allclose(u, RU / R, rtol=1e-15)
    u_all, n_all = fsl.favre_from_probes(str(path), H, real_bytes)  # to the end of the file
    assert n_all == 10


def _write_float_probes(path, H, steps, seed):
    rng = np.random.default_rng(seed)
    with open(path, "wb") as f:
        for step in steps:
            f.write(np.int32(step).tobytes())
            for _ in range(3):
                f.write((1.0 + 0.1 * rng.random(H)).astype(np.float32).tobytes())
                f.write((50.0 + 150.0 * rng.random(H)).astype(np.float32).tobytes())


@pytest.mark.parametrize("window", [(1, 9), (4, 7), (12, 12)])
def test_favre_profiles_equal_the_reference_program(fsl, oracle_lib, tmp_path, window):
    """The reference's own post-processor (favre-average-src/layer2_p.c,
    compiled unchanged into oracle/_ref/layer2_p) and fsl_favre_profiles on
    the same float probes file: probe1.dat .. probe3.dat byte for byte (float
    sums in file order, its text format).  The window ends before the file's
    last record: the reference's loop ends only on a step beyond step_end."""
    exe = os.path.join(os.path.dirname(oracle_lib.__file__), "_ref", "layer2_p")
    if not os.path.exists(exe):
        pytest.skip("the reference post-processor is not built (reference sources absent)")
    H = 9
    _write_float_probes(tmp_path / "probes.dat", H, list(range(1, 11)) + [13, 14], seed=5)
    ref_dir, mine = tmp_path / "ref", tmp_path / "mine"
    ref_dir.mkdir()
    mine.mkdir()
    (ref_dir / "probes.dat").write_bytes((tmp_path / "probes.dat").read_bytes())
    r = subprocess.run([exe], input="%d\n%d\n%d\n" % (window[0], window[1], H), text=True,
                       capture_output=True, cwd=ref_dir, timeout=30)
    assert r.returncode == 0, r.stdout[-500:]
    n = fsl.favre_profiles(str(tmp_path / "probes.dat"), H, window[0], window[1], str(mine))
    assert n == sum(1 for s in list(range(1, 11)) + [13, 14] if window[0] <= s <= window[1])
    for st in (1, 2, 3):
        a = (mine / ("probe%d.dat" % st)).read_bytes()
        assert a == (ref_dir / ("probe%d.dat" % st)).read_bytes(), st
        assert a.startswith(b"%d\n1\n" % (H + 2))


def test_stage_operation_counts():
    """The bench's per-cell-stage arithmetic (its compute roof) is the count
    the instrumented arithmetic templates give, for the fused kernel's
    composition; the reference's own composition (velocities per face)
    costs more divisions."""
    import json
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = os.path.join(root, "freeshearlayer_b200", "_build", "flopcount")
    if not os.path.exists(exe):
        subprocess.run(["make", "-C", os.path.join(root, "freeshearlayer_b200"), exe], check=True,
                       stdout=subprocess.DEVNULL)
    counts = json.loads(subprocess.run([exe], check=True, capture_output=True, text=True).stdout)
    sys.path.insert(0, root)
    import bench
    for prec, name in ((0, "fused"), (1, "fused_fp32")):
        got = counts[name]
        assert {k: got[k] for k in bench.STAGE_OPS[prec]} == bench.STAGE_OPS[prec], name
        assert got["flops"] == bench.STAGE_FLOPS[prec], name
    fused, ref = counts["fused"], counts["reference"]
    assert ref["div"] > fused["div"] and ref["flops"] > fused["flops"]
    # the FP32 bulk's regrouped sweeps and paired limiter do less of both
    assert counts["fused_fp32"]["flops"] < fused["flops"] and counts["fused_fp32"]["cmp"] < fused["cmp"]
    # the three face fluxes differ only in their permutation
    assert counts["face_x"] == counts["face_y"] == counts["face_z"]
