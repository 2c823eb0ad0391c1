"""The bench's placement of the e2e host buffers on the GPU's NUMA node, on the
CPU: a fake sysfs tree and fake affinity calls stand in for the box."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


class FakeProps:
    pci_domain_id = 0
    pci_bus_id = 0x9B
    pci_device_id = 0


def fake_box(tmp_path, monkeypatch, cpulist, allowed):
    dev = tmp_path / "0000:9b:00.0"
    dev.mkdir()
    (dev / "local_cpulist").write_text(cpulist + "\n")
    import torch
    monkeypatch.setattr(torch.cuda, "get_device_properties", lambda d: FakeProps())
    state = {"aff": set(allowed), "calls": []}
    monkeypatch.setattr(os, "sched_getaffinity", lambda pid: set(state["aff"]))

    def setaff(pid, cpus):
        state["calls"].append(set(cpus))
        state["aff"] = set(cpus)
    monkeypatch.setattr(os, "sched_setaffinity", setaff)
    return state


def test_cpulist_format():
    assert bench.parse_cpulist("0-3,8,10-11\n") == {0, 1, 2, 3, 8, 10, 11}
    assert bench.parse_cpulist("5") == {5}
    assert bench.parse_cpulist("") == set()


def test_binds_to_the_gpu_node_and_restores(tmp_path, monkeypatch):
    state = fake_box(tmp_path, monkeypatch, "48-95,144-191", range(192))
    near = bench.NearGpu(0, sysfs=str(tmp_path)).__enter__()
    assert state["aff"] == set(range(48, 96)) | set(range(144, 192))
    assert "96 cores" in near.describe()
    near.__exit__(None, None, None)
    assert state["aff"] == set(range(192))


def test_keeps_the_affinity_inside_the_node(tmp_path, monkeypatch):
    state = fake_box(tmp_path, monkeypatch, "0-7", range(4))
    near = bench.NearGpu(0, sysfs=str(tmp_path)).__enter__()
    near.__exit__(None, None, None)
    assert state["calls"] == [] and state["aff"] == set(range(4))
    assert "every allowed core (4) is local" in near.describe()


def test_keeps_the_affinity_outside_the_node(tmp_path, monkeypatch):
    state = fake_box(tmp_path, monkeypatch, "8-15", range(4))
    near = bench.NearGpu(0, sysfs=str(tmp_path)).__enter__()
    near.__exit__(None, None, None)
    assert state["calls"] == [] and "unknown" in near.describe()


def test_without_sysfs_nothing_changes(tmp_path, monkeypatch):
    state = fake_box(tmp_path, monkeypatch, "0-3", range(8))
    near = bench.NearGpu(0, sysfs=str(tmp_path / "missing")).__enter__()
    near.__exit__(None, None, None)
    assert state["calls"] == [] and "unknown" in near.describe()
