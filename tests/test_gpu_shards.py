"""One diagram over several shards (apo2_options.shard_index / shard_count): each handle builds
the cells of one contiguous Morton range, and the shards' outputs in shard order must be the
whole diagram's output, bit for bit. The shards run one after another on one GPU here; on
several GPUs each would run on its own device with no exchange (every shard holds all sites)."""
import numpy as np
import pytest

from tests import helpers as H

pytestmark = pytest.mark.gpu


def _full(sites, **kw):
    import apo_b200
    a = apo_b200.AlgorithmGPU(sites, **kw)
    a.build()
    full = a.toHostFull(True)
    topo = a.toTopology()
    stats = a.stats()
    a.close()
    return full, topo, stats


@pytest.mark.parametrize("case,count", [("uni2k", 2), ("uni2k", 5), ("protein20k", 3), ("uniform_small", 4)])
def test_shards_concatenate_to_the_whole_diagram(case, count):
    sites = H.sites_for(case)
    full, topo, stats = _full(sites)
    parts = [_full(sites, shard=(s, count)) for s in range(count)]
    for name in ("vertices", "verticesId", "closedEdgesMin", "closedEdgesId"):
        whole = getattr(full, name)
        joined = np.concatenate([getattr(p[0], name) for p in parts])
        assert np.array_equal(joined, whole), name
    for name in ("quadrisectors", "trisectors", "bisectors"):
        whole = getattr(topo, name)
        joined = np.concatenate([getattr(p[1], name) for p in parts])
        assert np.array_equal(joined, whole), name
    assert sum(p[2]["buried"] for p in parts) == stats["buried"]
    assert sum(p[2]["vertex_records"] for p in parts) == stats["vertex_records"]
    assert all(p[2]["error_flags"] == 0 for p in parts)
    # a shard holds per-cell stores for its own cells only
    assert all(p[2]["device_bytes"] < stats["device_bytes"] for p in parts)


def test_shards_with_other_k_and_knn_steps():
    sites = H.sites_for("uni2k")
    full, _, _ = _full(sites, k=4, knnValidationStep=3)
    parts = [_full(sites, k=4, knnValidationStep=3, shard=(s, 2))[0] for s in range(2)]
    assert np.array_equal(np.concatenate([p.vertices for p in parts]), full.vertices)
    assert np.array_equal(np.concatenate([p.verticesId for p in parts]), full.verticesId)


def test_shard_arguments():
    import apo_b200
    sites = H.sites_for("prec1")
    with pytest.raises(apo_b200.Apo2Error):
        apo_b200.AlgorithmGPU(sites, shard=(2, 2))
    a = apo_b200.AlgorithmGPU(sites, shard=(1, 2))
    a.build()
    order = a.debug_array("indices")  # sorted -> original: shard 1 holds the upper half
    a.cell(int(order[-1]))
    with pytest.raises(apo_b200.Apo2Error):
        a.cell(int(order[0]))
    a.close()
