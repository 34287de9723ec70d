"""bench.py's reference arm (the oracle on the host cores) on small samples
of each workload kind: one JSON-ready record with the contract's keys, the
metric of the workload's own arm, and a positive rate."""
import argparse
import json

import pytest


@pytest.mark.parametrize("workload,sample", [("sphere-5120", 8), ("hs-fault-10k-r32", 2),
                                             ("hs-uneven-32", 1), ("small-mixed", 4)])
def test_reference_arm_record(workload, sample, monkeypatch):
    import bench
    # the mixed sphere workload's kind on a 5,120-triangle sphere
    monkeypatch.setitem(bench.WORKLOADS, "small-mixed",
                        dict(kind="single_mixed", level=4, ntarg=100, targets="box", iprec=2, err_iprecs=(1,)))
    args = argparse.Namespace(workload=workload, steps=1, warmup=0, ref_sample=sample)
    out = bench.run_reference(args, 0)
    json.dumps(out)
    assert out["impl"] == "reference" and out["value"] > 0 and out["unit"] == "triangle-evals/s"
    assert out["higher_is_better"] is True and out["config"]["workload"] == workload
    assert out["cpu_baseline"]["kind"] == "port" and out["cpu_baseline"]["value"] == out["value"]
    assert out["e2e"] == {"value": out["value"], "unit": out["unit"], "h2d_bytes_per_step": 0,
                          "d2h_bytes_per_step": 0}
    kind = bench.WORKLOADS[workload]["kind"]
    if kind == "single_mixed":
        assert out["metric"] == bench.SINGLE_MIXED_METRIC
    if kind in ("hsbatch", "uneven"):
        assert "image" in out["cpu_baseline"]["sample"]
    assert bench.run_reference(args, 1) is None
