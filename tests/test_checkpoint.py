"""Checkpoint format (asd2g_checkpoint_*), host side: the numpy writer and
the library's reader agree on the layout and the checksum, and the reader
refuses damaged or foreign files.  No GPU needed (asd2g_checkpoint_info only
reads the file)."""
import numpy as np
import pytest

from asd2_b200 import api
from asd2_b200 import checkpoint as CK


def _fields(nx, ny, seed=0):
    rng = np.random.default_rng(seed)
    return {k: rng.standard_normal((nx + 6, ny + 6)) for k in CK.FIELDS}


def test_numpy_round_trip(tmp_path):
    f = _fields(20, 12)
    p = tmp_path / "a.ck"
    CK.write(p, f, t=0.25, step=7, dt=1e-3)
    g, meta = CK.read(p)
    assert meta["nx"] == 20 and meta["ny"] == 12 and meta["step"] == 7 and meta["t"] == 0.25
    for k in CK.FIELDS:
        assert np.array_equal(g[k], f[k])


def test_library_reads_numpy_checkpoint(tmp_path):
    p = tmp_path / "b.ck"
    CK.write(p, _fields(16, 24, seed=3), t=1.5, step=42, dt=2e-4)
    info = api.checkpoint_info(p)
    assert info == dict(nx=16, ny=24, t=1.5, step=42, dt=2e-4)


@pytest.mark.parametrize("damage", ["payload", "magic", "truncate"])
def test_library_refuses_damaged_file(tmp_path, damage):
    p = tmp_path / "c.ck"
    CK.write(p, _fields(8, 8, seed=5))
    raw = bytearray(p.read_bytes())
    if damage == "payload":
        raw[128 + 8 * 17 + 3] ^= 0x10
    elif damage == "magic":
        raw[0:8] = b"NOTACKPT"
    else:
        raw = raw[:-8]
    p.write_bytes(bytes(raw))
    with pytest.raises(api.Asd2gError) as e:
        api.checkpoint_info(p)
    assert e.value.code == -7
    with pytest.raises(ValueError):
        CK.read(p)


def test_checksum_sees_swapped_words():
    a = np.arange(1, 9, dtype="<f8").tobytes()
    b = np.array([2, 1, 3, 4, 5, 6, 7, 8], dtype="<f8").tobytes()
    assert CK.checksum(a) != CK.checksum(b)


def test_missing_file(tmp_path):
    with pytest.raises(api.Asd2gError) as e:
        api.checkpoint_info(tmp_path / "nope.ck")
    assert e.value.code == -7


@pytest.mark.parametrize("claim", ["huge_side", "huge_consistent_payload"])
def test_library_refuses_header_claiming_huge_grid(tmp_path, claim):
    """A damaged or crafted header that claims an enormous grid is refused
    with ASD2G_E_IO before any size arithmetic can overflow or a buffer of
    the claimed size is allocated."""
    import struct
    p = tmp_path / "h.ck"
    CK.write(p, _fields(8, 8, seed=6))
    raw = bytearray(p.read_bytes())
    if claim == "huge_side":
        struct.pack_into("<i", raw, 16, 2 ** 31 - 4)
    else:  # sides within int range and a payload size consistent with them, but absent from the file
        nx = ny = 60000
        struct.pack_into("<ii", raw, 16, nx, ny)
        struct.pack_into("<Q", raw, 64, 5 * (nx + 6) * (ny + 6) * 8)
    p.write_bytes(bytes(raw))
    with pytest.raises(api.Asd2gError) as e:
        api.checkpoint_info(p)
    assert e.value.code == -7


def test_reader_fuzz(tmp_path):
    """Random damage to a valid checkpoint (a flipped bit anywhere, a random
    byte run, a cut at any length, trailing bytes): the library's reader and
    the numpy reader refuse every damaged file (-7 / ValueError; the checksum
    covers the header too), accept it only where the damage rewrote bytes
    with their own values, and never crash."""
    hyp = pytest.importorskip("hypothesis")
    from hypothesis import HealthCheck, given, settings
    from hypothesis import strategies as st

    p0 = tmp_path / "base.ck"
    CK.write(p0, _fields(7, 5, seed=9), t=0.5, step=3, dt=1e-3)
    base = p0.read_bytes()
    truth = dict(nx=7, ny=5, t=0.5, step=3, dt=1e-3)

    @settings(max_examples=300, deadline=None, derandomize=True,
              suppress_health_check=[HealthCheck.function_scoped_fixture])
    @given(kind=st.sampled_from(("bit", "run", "cut", "extend")), pos=st.integers(0, len(base) - 1),
           bit=st.integers(0, 7), run=st.binary(min_size=1, max_size=24))
    def check(kind, pos, bit, run):
        raw = bytearray(base)
        if kind == "bit":
            raw[pos] ^= 1 << bit
        elif kind == "run":
            raw[pos:pos + len(run)] = run
        elif kind == "cut":
            raw = raw[:pos]
        else:
            raw += run
        p = tmp_path / "fuzz.ck"
        p.write_bytes(bytes(raw))
        try:
            info = api.checkpoint_info(p)
        except api.Asd2gError as e:
            assert e.code == -7, e
            info = None
        try:
            CK.read(p)
            ok_np = True
        except ValueError:
            ok_np = False
        assert (info is not None) == ok_np == (bytes(raw) == base), (kind, pos, bit, run)
        if info is not None:
            assert info == truth
    check()
