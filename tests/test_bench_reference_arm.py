"""bench.py's CPU side on the CPU: every workload's CPU baseline (the
oracle on a bounded sample) runs on a small sample, and the reference arm
prints the contract's JSON fields for every workload, with the workload
name our arm uses."""

import argparse
import json

import numpy as np
import pytest

import bench

WORKLOADS = ("elasticity", "batched-heat", "transient-heat", "serving",
             "av-phasor", "av-transient")


def _check_baseline(c):
    assert c["value"] > 0 and c["seconds"] > 0 and c["cores"] >= 1
    assert c["kind"] == "port" and c["unit"] == "DOF/s" and c["sample"]


def test_cpu_baselines_small_samples():
    _check_baseline(bench.cpu_baseline((4, 1, 1)))
    ns, ks = bench.batch_draw(6)
    _check_baseline(bench.cpu_baseline_batched_heat(ns, ks, cap_n=5, count=2))
    _check_baseline(bench.cpu_baseline_transient_heat(n=4, n_steps=2))
    _check_baseline(bench.cpu_baseline_av(nb=2))
    _check_baseline(bench.cpu_baseline_avt(nb=2, steps=2))
    pytest.importorskip("torch")
    _check_baseline(bench.cpu_baseline_serving(count=2, cap_dofs=2000))


@pytest.mark.parametrize("workload", WORKLOADS)
def test_reference_arm_json(monkeypatch, workload):
    fake = {"value": 123.0, "unit": "DOF/s", "cores": 4, "kind": "port",
            "seconds": 0.5, "sample": "fake sample"}
    for name in ("cpu_baseline", "cpu_baseline_batched_heat", "cpu_baseline_transient_heat",
                 "cpu_baseline_serving", "cpu_baseline_av", "cpu_baseline_avt"):
        monkeypatch.setattr(bench, name, lambda *a, **k: dict(fake))
    monkeypatch.setattr(bench, "batch_draw", lambda *a, **k: ([], []))
    args = argparse.Namespace(workload=workload, steps=2, warmup=1, gpus=1)
    out = bench.run_reference(args, 0)
    json.dumps(out)
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data",
                "config", "cpu_baseline", "e2e"):
        assert key in out, key
    assert out["impl"] == "reference" and out["value"] == 123.0
    assert out["e2e"]["h2d_bytes_per_step"] == 0 and out["e2e"]["d2h_bytes_per_step"] == 0
    assert out["e2e"]["value"] == out["value"] and out["e2e"]["unit"] == out["unit"]
    want = {"elasticity": "tet10_elasticity_beam_80x10x10",
            "batched-heat": "batched_tet10_heat_512_meshes_n4to24",
            "transient-heat": f"transient_p1_heat_cn_box_{bench.TRANSIENT_N}cubed_"
                              f"{bench.TRANSIENT_STEPS}_steps",
            "serving": f"serving_stream_{bench.SERVE_REQUESTS}_requests_lambda200",
            "av-phasor": f"phasor_av_tet10_box_{bench.AV_N}cubed",
            "av-transient": f"transient_av_tet10_box_{bench.AV_N}cubed_{bench.AVT_STEPS}_cn_steps"}
    assert out["config"]["workload"] == want[workload]
    assert bench.run_reference(args, 1) is None
    np.testing.assert_allclose(out["ms_per_step"], 500.0)
