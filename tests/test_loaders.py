"""Site loaders (apo_b200/loaders.py): MMTF decoding against arrays encoded here with the
format's codecs, the reference's sample structures when APO_REFERENCE_ROOT points at a checkout
of the reference, and the benchmark-set text format."""
import os
import struct

import numpy as np
import pytest

from apo_b200 import loaders

SAMPLES = os.path.join(os.environ.get("APO_REFERENCE_ROOT", "/nonexistent"), "app", "common", "samples")


def _encode(codec: int, param: int, payload: bytes, length: int) -> bytes:
    return struct.pack(">iii", codec, length, param) + payload


def _recursive_int16(values):
    out = []
    for v in values:
        while v >= 32767:
            out.append(32767)
            v -= 32767
        while v <= -32768:
            out.append(-32768)
            v += 32768
        out.append(v)
    return np.asarray(out, dtype=">i2").tobytes()


def _coords(values, divisor=1000):
    ints = np.round(np.asarray(values) * divisor).astype(np.int64)
    deltas = np.diff(np.concatenate([[0], ints]))
    return _encode(10, divisor, _recursive_int16(deltas.tolist()), len(values))


def test_codecs_round_trip():
    vals = [1.5, 40000.0, -70000.25, 3.0]
    assert np.allclose(loaders.decode_array(_coords(vals)), vals)
    ints = np.array([5, 0, 2], dtype=">i4")
    assert np.array_equal(loaders.decode_array(_encode(4, 0, ints.tobytes(), 3)), [5, 0, 2])
    rl = np.array([7, 3, 9, 2], dtype=">i4")  # run-length pairs: 7 x3, 9 x2
    assert np.array_equal(loaders.decode_array(_encode(7, 0, rl.tobytes(), 5)), [7, 7, 7, 9, 9])
    assert np.array_equal(loaders.decode_array(_encode(8, 0, rl.tobytes(), 5)), np.cumsum([7, 7, 7, 9, 9]))


def test_mmtf_first_model_in_file_order():
    import msgpack
    groups = [{"elementList": ["N", "C", "O"], "atomNameList": ["N", "CA", "O"]},
              {"elementList": ["S", "Fe"], "atomNameList": ["SG", "FE"]}]
    xs = [1.0, 2.0, 3.0, 4.0, 5.0, 9.0, 9.5]  # two models: 5 atoms, then 2 atoms of model 2
    doc = {
        "xCoordList": _coords(xs), "yCoordList": _coords([0.0] * 7), "zCoordList": _coords([-1.0] * 7),
        "groupTypeList": _encode(4, 0, np.array([0, 1, 1], dtype=">i4").tobytes(), 3),
        "groupList": groups, "chainsPerModel": [1, 1], "groupsPerChain": [2, 1], "numAtoms": 7,
    }
    sites = loaders.load_mmtf(msgpack.packb(doc, use_bin_type=True))
    assert sites.shape == (5, 4)
    assert np.allclose(sites[:, 0], xs[:5]) and np.allclose(sites[:, 2], -1.0)
    assert np.allclose(sites[:, 3], [1.55, 1.70, 1.52, 1.80, 1.0])  # Fe has no Bondi radius


@pytest.mark.skipif(not os.path.isdir(SAMPLES), reason="reference samples not present")
def test_mmtf_reference_samples():
    s = loaders.load_mmtf(os.path.join(SAMPLES, "1AON.mmtf"))
    assert s.shape == (58870, 4)  # the atom count the reference's knn benchmark quotes
    assert np.isfinite(s).all() and s[:, 3].min() >= 1.0


def test_dataset_text(tmp_path):
    p = tmp_path / "set.txt"
    p.write_text("3\n0 1.1 2.2 3.3 0.5\n1\t4.0 5.0 6.0 1.25\n2 0.1 0.2 0.3 2.0\n")
    s = loaders.load_dataset(str(p))
    assert s.shape == (3, 4)
    assert s[0, 0] == float(np.float32(1.1)) and s[1, 3] == 1.25
    bad = tmp_path / "bad.txt"
    bad.write_text("2\n0 1 2 3 4\n")
    with pytest.raises(ValueError):
        loaders.load_dataset(str(bad))
