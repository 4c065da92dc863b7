"""The bench line's derived numbers on the CPU, from fake kernel timings:
the roofline object (algorithmic bytes of a launch over its mean CUDA-event
time, against the HBM peak; DRAM traffic from the committed ncu summary,
scaled by cells), the compute roof (counted flops over the same time,
against the vector peak at the sampled clock), and the whole-job rate."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402

NAMES = ["stage", "recon", "flux", "sgs", "evol", "bc", "cfl", "other"]


class _KT:
    ms = [27.5, 0.0, 0.0, 25.0, 0.0, 3.3, 0.07, 0.07]
    launches = [10, 0, 0, 20, 0, 20, 10, 2]


@pytest.mark.parametrize("prec", [0, 1])
def test_stage_roofline_and_compute_roof(prec):
    ncell = 512 * 256 * 256
    peaks = {"hbm_gbs": 6650.0, "source": "fallback"}
    roof, kms, kl = bench.stage_roofline(_KT(), NAMES, ncell, prec, peaks, None)
    avg_s = 27.5e-3 / 10
    want = bench.STAGE_BYTES[prec] * ncell / avg_s / 1e9
    assert roof["achieved"] == pytest.approx(want, rel=1e-4)
    assert roof["frac"] == pytest.approx(want / 6650.0, abs=1e-4)
    assert roof["bound"] == "hbm" and roof["unit"] == "GB/s" and roof["launches"] == 10
    per_cell, where = bench.profiled_traffic(prec)
    if per_cell is not None:
        assert roof["traffic"] == pytest.approx(per_cell * ncell)
        assert where in roof["traffic_note"]
        assert 100.0 < per_cell < 200.0               # near the algorithmic bytes, not re-read
    assert kl["stage"] == 10 and kms["sgs"] == 25.0
    cr = bench.compute_roof(roof, prec, {"sm_mhz": 1965.0})
    lanes = 64 if prec == 0 else 128
    assert cr["peak"] == pytest.approx(148 * lanes * 2 * 1965e6 / 1e12, abs=0.01)
    assert cr["achieved"] == pytest.approx(bench.STAGE_FLOPS[prec] * ncell / avg_s / 1e12, rel=1e-3)


def test_whole_job_rate_is_weak_scaling():
    # every rank does the same units; the slowest rank's time counts
    assert bench.whole_job_rate(1000, 4, 20.0) == pytest.approx(4 * 1000 / 0.020)


def test_peaks_fall_back_without_the_measured_file(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    assert bench.measured_peaks() == {"hbm_gbs": 6650.0, "source": "fallback"}
    (tmp_path / "MEASURED_PEAKS.json").write_text('{"hbm_gbs": 7012.5, "bf16_tflops": 1600}')
    assert bench.measured_peaks() == {"hbm_gbs": 7012.5, "source": "measured"}


def test_gpus_flag_starts_that_many_ranks():
    """`bench.py --gpus 2` without a launcher starts two ranks under
    torch.distributed.run (gloo here, no GPU work): the line's n_gpus is 2 and
    its time the maximum over the ranks."""
    import json
    import subprocess
    env = dict(os.environ, FSL_BENCH_BACKEND="gloo", OMP_NUM_THREADS="1")
    env.pop("WORLD_SIZE", None)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--launcher-check"],
                       capture_output=True, text=True, timeout=180, env=env, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = json.loads(lines[0])
    assert line["n_gpus"] == 2 and line["ms_max"] == 11.0
    assert line["value"] == pytest.approx(2 * 1000 / 11e-3)


def test_gpus_flag_must_match_the_launcher():
    """Under a launcher that started another number of ranks, bench.py fails
    loudly instead of timing the wrong job."""
    import subprocess
    env = dict(os.environ, WORLD_SIZE="2", RANK="0", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "4", "--launcher-check"],
                       capture_output=True, text=True, timeout=60, env=env, cwd=ROOT)
    assert r.returncode != 0 and "WORLD_SIZE" in r.stderr


def test_cpu_ranges_and_binding_without_nvml_device():
    """The end-to-end leg's CPU binding: the range string it reports, and no
    binding (None) when NVML knows no such device (as on a host without a GPU)."""
    assert bench.cpu_ranges([0, 1, 2, 3, 8, 10, 11]) == "0-3,8,10-11"
    assert bench.cpu_ranges([5]) == "5"
    assert bench.cpu_ranges([]) == ""
    before = os.sched_getaffinity(0)
    assert bench.bind_near_gpu("GPU-00000000-0000-0000-0000-000000000000") is None
    assert os.sched_getaffinity(0) == before


def test_bind_near_gpu_uses_the_nvml_affinity(monkeypatch):
    """The end-to-end leg's binding takes the CPUs of NVML's affinity mask of
    the device (64 CPUs per word), restricted to those this process may use,
    and binds the process to them (NVML and the binding faked)."""
    import types
    calls = {}
    fake = types.SimpleNamespace(
        nvmlInit=lambda: None, nvmlShutdown=lambda: None,
        nvmlDeviceGetHandleByUUID=lambda u: calls.setdefault("uuid", u),
        # CPUs 0-3 and 66 of a 128-CPU host
        nvmlDeviceGetCpuAffinity=lambda h, n: [0b1111, 1 << 2][:n])
    monkeypatch.setitem(sys.modules, "pynvml", fake)
    monkeypatch.setattr(os, "cpu_count", lambda: 128)
    monkeypatch.setattr(os, "sched_getaffinity", lambda pid: {1, 2, 3, 66, 70})
    monkeypatch.setattr(os, "sched_setaffinity", lambda pid, cpus: calls.setdefault("bound", sorted(cpus)))
    assert bench.bind_near_gpu("GPU-abc") == [1, 2, 3, 66]
    assert calls == {"uuid": "GPU-abc", "bound": [1, 2, 3, 66]}
    assert bench.cpu_ranges([1, 2, 3, 66]) == "1-3,66"
