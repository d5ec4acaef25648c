"""Site loaders of the reference's applications, host side.

- `load_mmtf`: atoms of a macromolecular structure in MMTF format (the binary format of the
  RCSB), as the reference's `loadProtein` gives them (app/common/samples.cpp:10-61): the first
  model's atoms in file order (residue by residue), each as (x, y, z, van der Waals radius of its
  element), radius 1.0 for elements without one. The reference reads the file through chemfiles,
  which is not available here; this module decodes MMTF itself (MessagePack container, the
  format's binary array codecs) and takes radii from Bondi's table (A. Bondi, J. Phys. Chem. 68,
  441 (1964)), the table behind the radii of the protein-like generator.
- `load_dataset`: the text format of the sphere benchmark set the reference reads
  (app/common/samples.cpp:87-127): a count line, then "index x y z r" per line, parsed in single
  precision as the reference parses it.
"""
from __future__ import annotations

import struct

import numpy as np

# Bondi (1964) van der Waals radii, Angstrom, with the common additions for ions and metals.
VDW_RADII = {
    "H": 1.20, "HE": 1.40, "C": 1.70, "N": 1.55, "O": 1.52, "F": 1.47, "NE": 1.54, "SI": 2.10,
    "P": 1.80, "S": 1.80, "CL": 1.75, "AR": 1.88, "AS": 1.85, "SE": 1.90, "BR": 1.85, "KR": 2.02,
    "TE": 2.06, "I": 1.98, "XE": 2.16, "LI": 1.82, "NA": 2.27, "MG": 1.73, "K": 2.75, "NI": 1.63,
    "CU": 1.40, "ZN": 1.39, "GA": 1.87, "PD": 1.63, "AG": 1.72, "CD": 1.58, "IN": 1.93, "SN": 2.17,
    "PT": 1.75, "AU": 1.66, "HG": 1.55, "TL": 1.96, "PB": 2.02, "U": 1.86,
}


def _header(data: bytes) -> tuple[int, int, int, bytes]:
    codec, length, param = struct.unpack(">iii", data[:12])
    return codec, length, param, data[12:]


def _recursive_index(values: np.ndarray) -> np.ndarray:
    """Integers split into runs of the 16-bit (or 8-bit) extreme values are summed back."""
    info = np.iinfo(values.dtype)
    out = []
    acc = 0
    for v in values.tolist():
        acc += v
        if v != info.max and v != info.min:
            out.append(acc)
            acc = 0
    return np.asarray(out, dtype=np.int64)


def _run_length(values: np.ndarray) -> np.ndarray:
    pairs = values.reshape(-1, 2)
    return np.repeat(pairs[:, 0], pairs[:, 1])


def decode_array(data):
    """One MMTF binary array (codecs 1-10 of the MMTF specification, version 1.0)."""
    if not isinstance(data, (bytes, bytearray)):
        return data
    codec, length, param, body = _header(bytes(data))
    if codec == 1:
        return np.frombuffer(body, dtype=">f4").astype(np.float32)
    if codec == 2:
        return np.frombuffer(body, dtype=">i1").astype(np.int32)
    if codec == 3:
        return np.frombuffer(body, dtype=">i2").astype(np.int32)
    if codec == 4:
        return np.frombuffer(body, dtype=">i4").astype(np.int32)
    if codec == 5:
        raw = np.frombuffer(body, dtype=f"S{param}")
        return [s.decode().rstrip("\x00") for s in raw]
    if codec == 6:
        return [chr(c) if c else "" for c in _run_length(np.frombuffer(body, dtype=">i4"))]
    if codec == 7:
        return _run_length(np.frombuffer(body, dtype=">i4")).astype(np.int32)
    if codec == 8:
        return np.cumsum(_run_length(np.frombuffer(body, dtype=">i4"))).astype(np.int32)
    if codec == 9:
        return (_run_length(np.frombuffer(body, dtype=">i4")) / param).astype(np.float32)
    if codec == 10:
        ints = np.cumsum(_recursive_index(np.frombuffer(body, dtype=">i2").astype(np.int16)))
        return (ints / param).astype(np.float32)
    if codec == 11:
        return (np.frombuffer(body, dtype=">i2") / param).astype(np.float32)
    if codec == 12:
        return (_recursive_index(np.frombuffer(body, dtype=">i2").astype(np.int16)) / param).astype(np.float32)
    if codec == 13:
        return (_recursive_index(np.frombuffer(body, dtype=">i1").astype(np.int8)) / param).astype(np.float32)
    if codec == 14:
        return _recursive_index(np.frombuffer(body, dtype=">i2").astype(np.int16)).astype(np.int32)
    if codec == 15:
        return _recursive_index(np.frombuffer(body, dtype=">i1").astype(np.int8)).astype(np.int32)
    raise ValueError(f"unknown MMTF codec {codec}")


def _key(d: dict, name: str):
    v = d.get(name)
    if v is None:
        v = d.get(name.encode())
    return v


def load_mmtf(path_or_bytes) -> np.ndarray:
    """(n, 4) float64 sites (x, y, z, r) of the first model of an MMTF file, atoms in file order."""
    import msgpack
    data = path_or_bytes
    if not isinstance(data, (bytes, bytearray)):
        with open(path_or_bytes, "rb") as f:
            data = f.read()
    top = msgpack.unpackb(data, raw=False, strict_map_key=False)
    x = decode_array(_key(top, "xCoordList"))
    y = decode_array(_key(top, "yCoordList"))
    z = decode_array(_key(top, "zCoordList"))
    group_types = decode_array(_key(top, "groupTypeList"))
    group_list = _key(top, "groupList")
    chains_per_model = list(_key(top, "chainsPerModel"))
    groups_per_chain = list(_key(top, "groupsPerChain"))
    # the first model: its chains' groups, in order
    first_groups = int(sum(groups_per_chain[:chains_per_model[0]])) if chains_per_model else len(group_types)
    elements = []
    for g in range(first_groups):
        gt = group_list[int(group_types[g])]
        elements.extend(_key(gt, "elementList"))
    n = len(elements)
    radii = np.array([VDW_RADII.get(str(e).upper(), 1.0) for e in elements], dtype=np.float64)
    out = np.empty((n, 4), dtype=np.float64)
    out[:, 0] = x[:n]
    out[:, 1] = y[:n]
    out[:, 2] = z[:n]
    out[:, 3] = radii
    return out


def load_dataset(path: str) -> np.ndarray:
    """(n, 4) sites of a benchmark-set text file: a count line, then "index x y z r" lines,
    each value rounded to single precision as the reference's parser does."""
    rows = []
    with open(path) as f:
        count = int(f.readline().split()[0])
        for line in f:
            tokens = line.replace("\t", " ").split()
            if len(tokens) < 5:
                continue
            rows.append([float(np.float32(t)) for t in tokens[1:5]])
    out = np.asarray(rows, dtype=np.float64).reshape(-1, 4)
    if out.shape[0] != count:
        raise ValueError(f"{path}: {out.shape[0]} sites for a count of {count}")
    return out
