"""Host logic of bench.py that needs no GPU: the traffic figure of the
roofline follows the workload's view count and is dropped for other volume
or detector sizes, and the reference-CUDA comparison reports itself
unavailable, without touching a device, when the reference's installation
is absent."""

import json

import bench


def test_forward_traffic_scales_with_views_and_only_for_the_nominal_shapes():
    bench.parse_args([])
    full = bench.FWD_DRAM_BYTES["target512"]
    assert full is not None and bench.WORKLOAD["A"] == 720
    assert bench.forward_traffic(bench.WORKLOAD, 720) == full
    bench.parse_args(["--views", "48"])
    assert bench.forward_traffic(bench.WORKLOAD, 48) == full * 48 / 720
    bench.parse_args(["--volume", "256"])
    assert bench.forward_traffic(bench.WORKLOAD, 720) is None
    bench.parse_args(["--workload", "fdk256", "--detector", "512"])
    assert bench.forward_traffic(bench.WORKLOAD, 360) is None
    bench.parse_args([])


def test_refcuda_unavailable_without_the_reference_install(tmp_path, monkeypatch, capsys):
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    assert bench.load_reference_cuda() is None
    args = bench.parse_args(["--workload", "refcuda"])
    assert bench.run_refcuda(args) == 0
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["workload"] == "refcuda" and "not installed" in line["unavailable"]
