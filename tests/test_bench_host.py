"""Host-side checks of bench.py that need no GPU: the multi-rank dispatch and the
reference arm, which times the oracle port on the workload's own grid."""

import json

import pytest

import bench


def test_multi_rank_default_is_the_element_partition(monkeypatch):
    """With more than one rank the bench partitions the workload's elements over the
    ranks (face-trace exchange before every stage) unless --replicas is given."""
    called = []
    monkeypatch.setattr(bench, "run_sharded", lambda args, w: called.append(w["K"]) or 0)
    monkeypatch.setenv("WORLD_SIZE", "2")
    assert bench.main(["--gpus", "2", "--steps", "1", "--warmup", "3"]) == 0
    assert called == [32]

    class Stop(Exception):
        pass

    def stop(*a, **k):
        raise Stop()

    import torch
    import torch.distributed

    monkeypatch.setattr(bench, "load_product", stop)
    monkeypatch.setattr(torch.distributed, "init_process_group", stop)
    monkeypatch.setattr(torch.cuda, "set_device", lambda *a: None)
    with pytest.raises(Stop):
        bench.main(["--gpus", "2", "--replicas", "--steps", "1", "--warmup", "3"])
    assert called == [32]


def test_reference_arm_times_the_workload_grid(capsys, monkeypatch):
    monkeypatch.delenv("RANK", raising=False)
    assert bench.main(["--impl", "reference", "--workload", "adv2d_weak_n4_16_fp64", "--steps", "3",
                       "--warmup", "5"]) == 0
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["config"]["elements"] == 16 * 16 and line["config"]["nodes"] == 16 * 16 * 25
    assert line["timed_steps"] == 3 and line["steps"] == 3
    assert line["cpu_baseline"]["value"] == line["value"]
    assert "16^2-element" in line["cpu_baseline"]["sample"]


def test_launch_count_of_the_cluster_step_kernel():
    """One lsrk54_steps call is one launch on the cluster step kernel, and the stage (and
    mortar) kernels of every step otherwise (rb200_get_info: info[6] a step, info[9] the
    cluster's CTAs)."""
    import types

    cluster = types.SimpleNamespace(cluster_ctas=13, pipelined_ctas=0, geometry="affine", info=[2, 5, 1, 256, 0, 0, 5, 32, 0, 13])
    stages = types.SimpleNamespace(cluster_ctas=0, pipelined_ctas=444, geometry="affine", info=[3, 8, 5, 32768, 0, 0, 5, 152, 444, 0])
    assert bench.timed_launches(cluster, 100) == 1
    assert bench.timed_launches(stages, 20) == 100
    w = bench.WORKLOADS["adv2d_weak_n4_16_fp64"]
    assert bench.kernel_name(w, cluster).startswith("cluster_adv_steps_kernel")
    assert bench.kernel_name(bench.WORKLOADS["euler3d_kg_n7_32_fp64"], stages).startswith("pipelined_stage_kernel")
