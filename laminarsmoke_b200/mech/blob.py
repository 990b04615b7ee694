"""Packed mechanism blob: the file the C-ABI loads (``lsg_mech_load_blob``).

Layout (little endian, every payload 8-byte aligned)::

    char[8]  magic "LSMECH01"
    u32      number of arrays
    u32      reserved (0)
    repeat:
        char[32] name (NUL padded)
        u32      dtype   (0 = float64, 1 = int32)
        u32      reserved
        u64      element count
        payload  (count * itemsize bytes, then zero padding to 8 bytes)

The species names travel as one int32 array of UTF-8 bytes separated by NUL
(``species_names``) so the blob stays a flat list of numeric arrays.
"""
from __future__ import annotations

import struct
from typing import Dict, List

import numpy as np

MAGIC = b"LSMECH01"
_DT = {0: np.float64, 1: np.int32}


def _names_to_array(names: List[str]) -> np.ndarray:
    raw = b"\0".join(n.encode("utf-8") for n in names) + b"\0"
    return np.frombuffer(raw, dtype=np.uint8).astype(np.int32)


def _array_to_names(a: np.ndarray) -> List[str]:
    raw = bytes(a.astype(np.uint8).tolist())
    return [s.decode("utf-8") for s in raw.split(b"\0")[:-1]]


def pack(arrays: Dict[str, np.ndarray], species: List[str]) -> bytes:
    items = dict(arrays)
    items["species_names"] = _names_to_array(species)
    out = bytearray()
    out += MAGIC
    out += struct.pack("<II", len(items), 0)
    for name, arr in items.items():
        arr = np.asarray(arr)
        if arr.dtype == np.float64:
            code = 0
        elif arr.dtype == np.int32:
            code = 1
        else:
            raise TypeError(f"{name}: unsupported dtype {arr.dtype}")
        nb = name.encode("ascii")
        if len(nb) >= 32:
            raise ValueError(f"array name too long: {name}")
        out += nb + b"\0" * (32 - len(nb))
        out += struct.pack("<IIQ", code, 0, arr.size)
        payload = np.ascontiguousarray(arr.ravel()).tobytes()
        out += payload
        out += b"\0" * ((-len(payload)) % 8)
    return bytes(out)


def unpack(data: bytes):
    if data[:8] != MAGIC:
        raise ValueError("not a packed mechanism (bad magic)")
    n, _ = struct.unpack_from("<II", data, 8)
    pos = 16
    arrays: Dict[str, np.ndarray] = {}
    for _ in range(n):
        name = data[pos:pos + 32].split(b"\0")[0].decode("ascii")
        code, _, count = struct.unpack_from("<IIQ", data, pos + 32)
        pos += 48
        dt = np.dtype(_DT[code])
        nbytes = count * dt.itemsize
        arrays[name] = np.frombuffer(data, dtype=dt, count=count, offset=pos).copy()
        pos += nbytes + ((-nbytes) % 8)
    species = _array_to_names(arrays.pop("species_names"))
    return arrays, species
