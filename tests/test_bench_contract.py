"""bench.py's output contract, checked on the CPU: the reference arm's JSON line, the figures the
GPU arm reads from the committed ncu summary, the peak denominators and the clock summary."""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
import bench  # noqa: E402  (the repo root is on sys.path via conftest)


def _run(*args, env=None):
    e = dict(os.environ, OMP_NUM_THREADS="2")
    e.update(env or {})
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), *map(str, args)], capture_output=True,
                          text=True, env=e, cwd=ROOT, timeout=600)


def test_reference_arm_prints_one_contract_line(oracle_mod):
    r = _run("--impl", "reference", "--n", 64, "--steps", 2, "--warmup", 3, "--ref-solver-steps", 2)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC and d["unit"] == bench.UNIT and d["higher_is_better"] is True
    assert d["n_gpus"] == 1 and d["steps"] == 2 and d["warmup"] == 3 and d["dtype"] == "f64"
    assert d["config"] == bench.bench_config(64, 1)  # the same config as the GPU arm reports
    assert d["value"] > 0 and d["ms_per_step"] > 0
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["unit"] == bench.UNIT and cb["cores"] >= 1
    assert cb["kind"] in ("reference", "port") and "64^2" in cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": bench.UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    # 4 combos x 2 solver steps x 64^2 cells per bench step
    assert d["value"] == pytest.approx(2 * 4 * 2 * 64 * 64 / (d["ms_per_step"] * 2 / 1e3), rel=1e-9)


def test_reference_arm_runs_on_rank_zero_only():
    r = _run("--impl", "reference", "--n", 64, "--steps", 1, "--warmup", 3,
             env={"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r.returncode == 0 and r.stdout.strip() == "", (r.returncode, r.stdout, r.stderr)


def test_roofline_figures_come_from_the_committed_summary():
    assert bench.profiled_traffic() == 25213952.0  # DRAM bytes per stage-2 launch at 512^2
    assert bench.profiled_traffic() == pytest.approx(bench.STAGE_BYTES[2] * 512 * 512, rel=0.01)
    assert 0.0 < bench.profiled("fp64_pipe_active_stage2") < 1.0
    assert bench.profiled("no_such_figure") is None
    # the stepper's figures: DRAM bytes per step (L2-resident grid: far below the 160 B/cell of HBM
    # traffic), executed FP64 flops per cell-step and FP64 pipe activity
    assert 0 < bench.profiled("traffic_bytes_per_step_stepper") < 160 * 512 * 512
    assert 500 < bench.profiled("fp64_flops_per_cell_step") < 3000
    assert 0.0 < bench.profiled("fp64_pipe_active_stepper") < 1.0
    r = bench.fp64_roofline(512, 0.0415, per="step")  # a 41.5 us step at 512^2
    assert r["achieved"] == pytest.approx(bench.profiled("fp64_flops_per_cell_step") * 512 * 512 / 41.5e-6 / 1e12)


def test_peak_denominator_measured_or_fallback(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    assert bench.measured_peaks() == (6650.0, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6538.2, "bf16_tflops": 1590.0}))
    assert bench.measured_peaks() == (6538.2, "measured")


def test_clock_summary_reads_median_and_reasons(tmp_path):
    c = bench.Clocks(0)
    c.path = str(tmp_path / "clocks.csv")
    rows = ["1965, 1965, 812.4, Not Active, Not Active, Not Active, Not Active",
            "1950, 1965, 990.1, Not Active, Not Active, Not Active, Active",
            "[N/A], 1965, 0.0, Not Active, Not Active, Not Active, Not Active",  # unreadable sample: skipped
            "1965, 1965, 1001.0, Not Active, Not Active, Not Active, Active"]
    Path(c.path).write_text("\n".join(rows) + "\n")
    s = c.summary()
    assert s == {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}
    assert not os.path.exists(c.path)


def test_clock_summary_flags_slowdowns(tmp_path):
    c = bench.Clocks(0)
    c.path = str(tmp_path / "clocks.csv")
    Path(c.path).write_text("1200, 1965, 700.0, Active, Not Active, Active, Not Active\n")
    assert c.summary()["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"]


def test_fp64_roofline_of_the_stage_kernel(tmp_path, monkeypatch):
    r = bench.fp64_roofline(512, 0.0238)  # a 23.8 us stage-1 launch at 512^2
    assert r["unit"] == "TFLOP/s" and r["flops_per_cell"] == 548.0 and r["peak"] == 36.2
    assert r["achieved"] == pytest.approx(548 * 512 * 512 / 23.8e-6 / 1e12)  # ~6.04 TFLOP/s
    assert r["frac"] == pytest.approx(r["achieved"] / 36.2) and 0.1 < r["frac"] < 0.25
    assert r["pipe_active_ncu"] == 0.433
    assert bench.fp64_roofline(512, 0.0) is None  # no timed launches
    monkeypatch.setattr(bench, "ROOT", tmp_path)  # no committed summary: no figure, no error
    assert bench.fp64_roofline(512, 0.0238) is None
    assert bench.profiled_traffic() is None


def _reduce_worker(rank, world, port, out_dir):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    import bench as b
    out = b.reduce_over_ranks(10.0 + 5.0 * rank, 1000.0 * (rank + 1), 7 + rank, "cpu")
    (Path(out_dir) / f"r{rank}.json").write_text(json.dumps(list(out)))
    dist.destroy_process_group()


def test_timing_is_the_max_over_ranks_and_work_the_sum(tmp_path):
    """The N > 1 reduction of bench.py's timed regions (time: max; work and launches: sum), as 2 gloo
    ranks on the CPU."""
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(_reduce_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    for r in range(2):
        assert json.loads((tmp_path / f"r{r}.json").read_text()) == [15.0, 3000.0, 15]


def test_clock_sampling_follows_the_device_mask(monkeypatch):
    monkeypatch.delenv("CUDA_VISIBLE_DEVICES", raising=False)
    assert bench.smi_id(0) == "0" and bench.smi_id(3) == "3"
    monkeypatch.setenv("CUDA_VISIBLE_DEVICES", "5,2")
    assert bench.smi_id(0) == "5" and bench.smi_id(1) == "2"
    monkeypatch.setenv("CUDA_VISIBLE_DEVICES", "GPU-8f1e, GPU-77aa")
    assert bench.smi_id(1) == "GPU-77aa"
    assert bench.Clocks(0).index == "GPU-8f1e"


def test_a_tolerance_build_run_says_so_in_its_config():
    assert "build" not in bench.bench_config(512, 1)
    assert bench.bench_config(512, 1, "tolerance")["build"].startswith("tolerance: FMA contraction")
    assert {k: v for k, v in bench.bench_config(512, 1, "tolerance").items() if k != "build"} == bench.bench_config(512, 1)
