"""Reader and writer of the asd2g checkpoint format in numpy, for processes
without a GPU (the CPU restatement, analysis scripts).  The layout is the one
asd2g_checkpoint_save writes: a 128-byte little-endian header

    char magic[8] = "ASD2GCK1"; u32 version = 2; u32 header_bytes = 128;
    i32 nx, ny, nbc (= 3), precision; f64 t, dt; i64 step;
    u32 nfields (= 5), field_bits; u64 payload_bytes; u64 checksum;
    48 zero bytes

followed by the padded (nx+6) x (ny+6) FP64 arrays LS, U, V, PS, P.  The
checksum is the weighted word sum  sum_i w_i (2 i + 1)  mod 2^64 over the
little-endian 64-bit words w_i of the header (its checksum field read as 0;
words 0-15) followed by the payload (words 16 on): any changed word, header
included, or any exchange of two different words changes it.
"""
from __future__ import annotations

import numpy as np

MAGIC = b"ASD2GCK1"
FIELDS = ("ls", "u", "v", "ps", "p")
FIELD_IDS = {"ls": 0, "u": 1, "v": 2, "ps": 3, "p": 4}  # asd2g field ids (include/asd2g.h)
HEADER = np.dtype([("magic", "S8"), ("version", "<u4"), ("header_bytes", "<u4"), ("nx", "<i4"), ("ny", "<i4"),
                   ("nbc", "<i4"), ("precision", "<i4"), ("t", "<f8"), ("dt", "<f8"), ("step", "<i8"),
                   ("nfields", "<u4"), ("field_bits", "<u4"), ("payload_bytes", "<u8"), ("checksum", "<u8"),
                   ("reserved", "V48")])
assert HEADER.itemsize == 128


def checksum(payload: bytes, first: int = 0) -> int:
    """Weighted word sum of 64-bit words (a multiple of 8 bytes), mod 2^64, the
    word index counted from `first`."""
    w = np.frombuffer(payload, dtype="<u8")
    k = (np.arange(w.size, dtype=np.uint64) + np.uint64(first)) * np.uint64(2) + np.uint64(1)
    with np.errstate(over="ignore"):
        return int(np.sum(w * k, dtype=np.uint64))


def file_checksum(header: np.ndarray, payload: bytes) -> int:
    """The file's checksum: the header with its checksum field zeroed (words
    0-15), then the payload (words 16 on)."""
    z = np.frombuffer(header.tobytes(), dtype=HEADER).copy()
    z["checksum"] = 0
    hw = HEADER.itemsize // 8
    return (checksum(z.tobytes()) + checksum(payload, hw)) % (1 << 64)


def write(path, fields: dict, t=0.0, step=0, dt=0.0, precision=0):
    """fields: name -> padded (nx+6, ny+6) float64 array for every name of FIELDS."""
    arrs = [np.ascontiguousarray(fields[k], dtype="<f8") for k in FIELDS]
    gx, gy = arrs[0].shape
    payload = b"".join(a.tobytes() for a in arrs)
    h = np.zeros((), dtype=HEADER)
    h["magic"], h["version"], h["header_bytes"] = MAGIC, 2, 128
    h["nx"], h["ny"], h["nbc"], h["precision"] = gx - 6, gy - 6, 3, precision
    h["t"], h["dt"], h["step"] = t, dt, step
    h["nfields"] = len(FIELDS)
    h["field_bits"] = sum(1 << FIELD_IDS[k] for k in FIELDS)
    h["payload_bytes"] = len(payload)
    h["checksum"] = file_checksum(h, payload)
    with open(path, "wb") as f:
        f.write(h.tobytes())
        f.write(payload)


MAX_SIDE = 1 << 20  # the largest nx / ny a reader accepts (as the library's)


def read(path):
    """(fields dict, header dict) after the checks the library's reader makes:
    magic, version, header size, grid sides within [1, MAX_SIDE], three ghost
    layers, five fields, payload size and checksum."""
    with open(path, "rb") as f:
        raw = f.read()
    if len(raw) < HEADER.itemsize:
        raise ValueError(f"{path}: short header")
    h = np.frombuffer(raw[:128], dtype=HEADER)[0]
    if bytes(h["magic"]) != MAGIC or int(h["version"]) != 2 or int(h["header_bytes"]) != HEADER.itemsize:
        raise ValueError(f"{path}: not an asd2g checkpoint")
    nx, ny = int(h["nx"]), int(h["ny"])
    if not (1 <= nx <= MAX_SIDE and 1 <= ny <= MAX_SIDE) or int(h["nbc"]) != 3 or int(h["nfields"]) != len(FIELDS):
        raise ValueError(f"{path}: inconsistent sizes")
    g = (nx + 6) * (ny + 6)
    payload = raw[128:]
    if len(payload) != int(h["payload_bytes"]) or len(payload) != 8 * g * len(FIELDS):
        raise ValueError(f"{path}: inconsistent sizes")
    if file_checksum(h, payload) != int(h["checksum"]):
        raise ValueError(f"{path}: checksum mismatch")
    data = np.frombuffer(payload, dtype="<f8").reshape(len(FIELDS), nx + 6, ny + 6)
    fields = {k: data[i].copy() for i, k in enumerate(FIELDS)}
    meta = {k: (h[k].item() if k != "magic" else bytes(h[k])) for k in ("nx", "ny", "t", "dt", "step", "precision")}
    return fields, meta
