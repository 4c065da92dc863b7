"""Driver files on the GPU path: backup.dat written and restored in the
reference's layout (src/finalize.c, src/initialize.c:133-158), Probes()
records (src/probes.c) and the device-side Favre average."""
import numpy as np
import pytest

from tests.helpers import random_state, spatial_params, temporal_params

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fsl():
    import freeshearlayer_b200 as fsl
    return fsl


@pytest.mark.parametrize("real_bytes", [8, 4])
def test_backup_roundtrip_and_layout(fsl, tmp_path, real_bytes):
    p = spatial_params(L=12, H=8, D=6)
    a = fsl.Domain(p)
    a.upload_state(random_state(p, 4))
    a.step(3)
    path = tmp_path / "backup.dat"
    a.write_backup(str(path), real_bytes)
    st, info = a.download_state(), a.info()
    raw = path.read_bytes()
    n = st.size
    dt = np.float32 if real_bytes == 4 else np.float64
    fields = np.frombuffer(raw[:n * real_bytes], dt)
    np.testing.assert_array_equal(fields, st.astype(dt))          # per (i, j): DEP rows of U1..U5
    assert np.frombuffer(raw[n * real_bytes:(n + 1) * real_bytes], dt)[0] == dt(info.deltaT)
    assert np.frombuffer(raw[(n + 1) * real_bytes:], np.int32)[0] == info.step == 3
    b = fsl.Domain(p)
    b.read_backup(str(path), real_bytes)
    ib = b.info()
    assert ib.step == 3 and ib.deltaT == float(dt(info.deltaT))
    np.testing.assert_array_equal(b.download_state(), st.astype(dt).astype(np.float64))
    if real_bytes == 8:  # FP64 restart continues bit-identically
        a.step(2)
        b.step(2)
        np.testing.assert_array_equal(a.download_state(), b.download_state())


def test_backup_size_mismatch_is_an_error(fsl, tmp_path):
    p = spatial_params(L=12, H=8, D=6)
    a = fsl.Domain(p)
    a.upload_state(random_state(p, 4))
    path = tmp_path / "backup.dat"
    a.write_backup(str(path), 8)
    q = fsl.Domain(spatial_params(L=12, H=8, D=7))
    with pytest.raises(fsl.FslError) as e:
        q.read_backup(str(path), 8)
    assert e.value.code == -6


def test_probes_and_favre(fsl, tmp_path):
    p = temporal_params(L=16, H=12, D=10)
    s, _ = fsl.temporal_state(p, 0.4, 1.0, 1e-2, 7)
    d = fsl.Domain(p)
    d.upload_state(s)
    path = tmp_path / "probes.dat"
    d.favre_reset()
    for _ in range(4):
        d.step(1)
        d.write_probes(str(path), 8)
        d.favre_accumulate()
    # the record of the last step against the state
    L, H, D = p["LEN"], p["HIG"], p["DEP"]
    st = d.download_state().reshape(L, H, 5, D)
    rows = d.probe_rows()
    k = D // 2 + 1
    for sidx, i in enumerate((L // 2, 3 * L // 4, L)):
        np.testing.assert_array_equal(rows[sidx, 0], st[i - 1, :, 0, k - 1])
        np.testing.assert_array_equal(rows[sidx, 1], st[i - 1, :, 1, k - 1])
    raw = np.frombuffer(path.read_bytes(), np.uint8)
    rec = 4 + 6 * H * 8
    assert raw.size == 4 * rec
    assert np.frombuffer(raw[3 * rec:3 * rec + 4].tobytes(), np.int32)[0] == 4
    np.testing.assert_array_equal(np.frombuffer(raw[3 * rec + 4:4 * rec].tobytes(), np.float64), rows.ravel())
    u_dev, n_dev = d.favre_read()
    u_file, n_file = fsl.favre_from_probes(str(path), H, 8)
    assert n_dev == n_file == 4
    np.testing.assert_allclose(u_dev, u_file, rtol=1e-14)


def test_host_driver_run_and_restart(fsl, oracle_lib, tmp_path):
    """The ANSI-C driver (host/layer2_gpu.c) reads layer2.ini and the seed from
    stdin like src/layer2.c, appends a probes record per step and writes
    backup.dat; its state matches the oracle bit for bit, and a restart
    (Answer = 1) continues exactly (the deltaT the reference's reader skips is
    restored)."""
    import os
    import subprocess
    exe = os.path.join(os.path.dirname(fsl.__file__), "layer2_gpu")
    if not os.path.exists(exe):
        pytest.skip("layer2_gpu not built")
    # no disturbance amplitude: the driver re-seeds the disturbance RNG from
    # stdin on a restart (as src/layer2.c does), so only an undisturbed
    # inflow continues bit for bit
    p = spatial_params(L=12, H=8, D=6, numstep=4, Answer=0, Ua=0.0, Va=0.0, Wa=0.0)
    (tmp_path / "layer2.ini").write_text(oracle_lib.ini_text(p))
    seed = "%.12f\n" % p["seed_X"]
    r = subprocess.run([exe], input=seed, text=True, capture_output=True, cwd=tmp_path, timeout=120)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    o = oracle_lib.Oracle(p)
    o.set_state(fsl.initial_state(p))
    o.step(4)
    n = p["LEN"] * p["HIG"] * 5 * p["DEP"]
    raw = (tmp_path / "backup.dat").read_bytes()
    np.testing.assert_array_equal(np.frombuffer(raw[:8 * n], np.float64), o.state())
    assert (tmp_path / "probes.dat").stat().st_size == 4 * (4 + 6 * p["HIG"] * 8)
    frame = (tmp_path / "4.plt").read_text().splitlines()      # the end-of-run Output() frame
    assert len(frame) == 15 + p["LEN"] * p["HIG"] * p["DEP"] and frame[14].startswith("i=12, j=8, k=6")
    p2 = dict(p, numstep=6, Answer=1)
    (tmp_path / "layer2.ini").write_text(oracle_lib.ini_text(p2))
    r = subprocess.run([exe], input=seed, text=True, capture_output=True, cwd=tmp_path, timeout=120)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    o.step(2)
    raw = (tmp_path / "backup.dat").read_bytes()
    np.testing.assert_array_equal(np.frombuffer(raw[:8 * n], np.float64), o.state())
    assert np.frombuffer(raw[-4:], np.int32)[0] == 6


def test_output_frame_matches_oracle(fsl, oracle_lib, tmp_path):
    """Output()'s values (src/output.c) from the GPU state after steps equal
    the oracle's bit for bit, and the written Tecplot frame equals the one
    written from the oracle's values."""
    p = spatial_params(L=12, H=8, D=6)
    s = oracle_lib.spatial_initial_state(p)
    o = oracle_lib.Oracle(p)
    o.set_state(s)
    o.step(3)
    d = fsl.Domain(p)
    d.upload_state(s)
    d.step(3)
    a, b = d.output_fields(), o.output_fields()
    assert np.array_equal(a, b)
    d.write_tecplot(str(tmp_path / "gpu.plt"))
    fsl.tecplot_write(str(tmp_path / "orc.plt"), b)
    assert (tmp_path / "gpu.plt").read_bytes() == (tmp_path / "orc.plt").read_bytes()


def test_async_transfers_match_the_synchronous_ones(fsl):
    """Pipelined fsl_upload_state_async / fsl_step / fsl_download_state_async
    over three different inputs: every result equals that of the same
    sequence through the synchronous calls."""
    from tests.helpers import temporal_params
    import torch
    p = temporal_params(L=24, H=12, D=16)
    states = [fsl.temporal_state(fsl._as_params(p), 0.4, 1.0, 2e-2, 11 + q)[0] for q in range(3)]
    n = states[0].size
    ins = [torch.empty(n, dtype=torch.float64, pin_memory=True).numpy() for _ in range(3)]
    outs = [torch.empty(n, dtype=torch.float64, pin_memory=True).numpy() for _ in range(3)]
    for a, s in zip(ins, states):
        a[:] = s
    d = fsl.Domain(p)
    for q in range(3):
        d.upload_state_async(ins[q])
        d.step(2)
        d.download_state_async(outs[q])
    d.transfer_wait()
    d.close()
    # the same sequence with the synchronous calls (deltaT carries over)
    r = fsl.Domain(p)
    for q in range(3):
        r.upload_state(states[q])
        r.step(2)
        assert np.array_equal(outs[q], r.download_state()), q
    r.close()


def test_host_driver_headline_path(fsl, oracle_lib, tmp_path):
    """The ANSI-C driver runs the FP32 bulk with the learned closure (weights
    file, feature scales, judgements every 2 steps) from the optional
    layer2_gpu.ini beside an unchanged layer2.ini, starting from the temporal
    shear layer: its backup.dat equals the same steps through the library."""
    import os
    import subprocess
    exe = os.path.join(os.path.dirname(fsl.__file__), "layer2_gpu")
    if not os.path.exists(exe):
        pytest.skip("layer2_gpu not built")
    from tests.helpers import temporal_params
    p = temporal_params(L=24, H=16, D=16, Mc=0.5, Re=2000.0, numstep=5, Answer=0)
    (tmp_path / "layer2.ini").write_text(oracle_lib.ini_text(p))
    dU = 2.0 * 0.5 * np.sqrt(1.4e5)
    (tmp_path / "layer2_gpu.ini").write_text(
        "# the headline path\nprecision = fp32\nsgs = learned   \nsetup = temporal\ncfl = acoustic\n"
        "closure_weights = %s\nclosure_t_ref = %.17g\nclosure_len_ref = 1\njudge_every = 2\n"
        "judge_threshold = 0.02\ntemporal_state = 0.5 1.0 0.02 7\n" % (fsl.CLOSURE_WEIGHTS, 1.0 / dU))
    r = subprocess.run([exe], input="%.12f\n" % p["seed_X"], text=True, capture_output=True, cwd=tmp_path,
                       env=dict(os.environ, FSL_FRAMES="0", FSL_PROBES="0"), timeout=120)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    q = dict(p, precision=1, sgs=1)
    s, dU2 = fsl.temporal_state(q, 0.5, 1.0, 0.02, 7)
    d = fsl.Domain(q)
    d.upload_state(s)
    d.closure_set_scales(1.0 / dU, 1.0)
    d.closure_set_weights(fsl.closure_weights())
    d.closure_judge(2, 0.02)
    for _ in range(5):
        d.step(1)
        d.sync()
    n = p["LEN"] * p["HIG"] * 5 * p["DEP"]
    raw = (tmp_path / "backup.dat").read_bytes()
    np.testing.assert_array_equal(np.frombuffer(raw[:8 * n], np.float64), d.download_state())
    assert d.closure_stats().judgements == 3
    # an unknown option is refused with the line it came from
    (tmp_path / "layer2_gpu.ini").write_text("precision = fp16\n")
    r = subprocess.run([exe], input="0.3\n", text=True, capture_output=True, cwd=tmp_path, timeout=60)
    assert r.returncode != 0 and "layer2_gpu.ini:1" in r.stdout


def test_favre_profiles_from_gpu_probes_equal_the_reference_program(fsl, oracle_lib, tmp_path):
    """Probes records written from the GPU state in the reference's float
    format (fsl_write_probes, real_bytes 4) over 8 steps, post-processed by
    the reference's own program (favre-average-src/layer2_p.c) and by
    fsl_favre_profiles: the three profile files are byte-identical."""
    import os
    import subprocess
    exe = os.path.join(os.path.dirname(oracle_lib.__file__), "_ref", "layer2_p")
    if not os.path.exists(exe):
        pytest.skip("the reference post-processor is not built")
    p = spatial_params(L=16, H=10, D=8)
    d = fsl.Domain(p)
    d.upload_state(oracle_lib.spatial_initial_state(p))
    path = tmp_path / "probes.dat"
    for _ in range(8):
        d.step(1)
        d.write_probes(str(path), 4)
    d.close()
    ref_dir, mine = tmp_path / "ref", tmp_path / "mine"
    ref_dir.mkdir()
    mine.mkdir()
    (ref_dir / "probes.dat").write_bytes(path.read_bytes())
    r = subprocess.run([exe], input="2\n7\n%d\n" % p["HIG"], text=True, capture_output=True, cwd=ref_dir,
                       timeout=30)
    assert r.returncode == 0
    assert fsl.favre_profiles(str(path), p["HIG"], 2, 7, str(mine)) == 6
    for st in (1, 2, 3):
        assert (mine / ("probe%d.dat" % st)).read_bytes() == (ref_dir / ("probe%d.dat" % st)).read_bytes()
