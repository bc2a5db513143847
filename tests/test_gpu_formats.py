"""SEG-Y sample codec on the device against the oracle's restatement of the
format (bit-exact, IBM and IEEE), and the reference's own round-trip checks
(tests/test_io.py:49-115 of the reference) through the public API."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import ertm_oracle as orc

pytestmark = pytest.mark.gpu


def _make_shot(source_x=100.0, nrec=11, nt=64):
    from ertm_b200.types import ReceiverSpec, ShotRecord, SourceSpec
    x = np.linspace(0.0, 200.0, nrec)
    data = np.random.default_rng(int(source_x)).normal(size=(nt, nrec)).astype(np.float32)
    return ShotRecord(data=data, dt=4.0e-4, t=np.arange(nt, dtype=np.float64) * 4.0e-4,
                      receivers=ReceiverSpec(x=x, z=np.full(nrec, 20.0), component="p"),
                      source=SourceSpec(x=source_x, z=20.0, f0=20.0), components={"p": data})


def _awkward(ns, ntr, seed):
    """Random float32 bit patterns plus ±0, ±inf, NaN, denormals and IBM edge values."""
    bits = np.random.default_rng(seed).integers(0, 2 ** 32, ns * ntr, dtype=np.uint64).astype(np.uint32)
    x = bits.view(np.float32).copy()
    x[:12] = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 1e-45, -3e-39, 1.0, -118.625, 3.4e38, 5e-38, 0.15625],
                      dtype=np.float32)
    return x.reshape(ns, ntr)


@pytest.mark.parametrize("fmt", [1, 5])
def test_encode_bytes_equal_oracle_file(tmp_path, fmt):
    from ertm_b200 import segy
    shot = _make_shot(120.0, nrec=37, nt=70)
    shot.data[:] = _awkward(70, 37, fmt)
    shot.data[~np.isfinite(shot.data)] = 0.0            # a ShotRecord holds finite samples only
    path = segy.write_segy_shot(shot, tmp_path / "s.sgy", fmt=fmt)
    heads = [{"SourceX": 120, "SourceY": 20, "GroupX": int(round(float(g))), "GroupY": 20, "SourceGroupScalar": 1,
              "offset": int(round(abs(float(g) - 120.0))), "FieldRecord": 1, "TraceNumber": k + 1,
              "TRACE_SAMPLE_COUNT": 70, "TRACE_SAMPLE_INTERVAL": 400} for k, g in enumerate(shot.receivers.x)]
    assert path.read_bytes() == orc.segy_bytes(shot.data, heads, 400, fmt, "ERTM shot 120.0/20.0")


@pytest.mark.parametrize("fmt", [1, 5])
def test_decode_bit_exact_with_permutation(tmp_path, fmt):
    from ertm_b200 import segy
    ns, ntr = 93, 77                                    # ragged against the 32×32 tiles
    rec = _awkward(ns, ntr, 10 + fmt)
    ibm_words = np.random.default_rng(7).integers(0, 2 ** 32, ns * ntr, dtype=np.uint64).astype(np.uint32)
    heads = [{"TraceNumber": k + 1, "TRACE_SAMPLE_COUNT": ns} for k in range(ntr)]
    blob = bytearray(orc.segy_bytes(rec, heads, 1000, fmt, "t"))
    if fmt == 1:                                        # arbitrary IBM words, unnormalised ones included
        for k in range(ntr):
            off = 3600 + k * (240 + 4 * ns) + 240
            blob[off:off + 4 * ns] = ibm_words.reshape(ns, ntr)[:, k].astype(">u4").tobytes()
    p = tmp_path / "d.sgy"
    p.write_bytes(bytes(blob))
    _, _, want = orc.segy_parse(bytes(blob))
    sf = segy.open_segy(p)
    cols = [np.array([5, 0, 76, 3]), np.arange(ntr)[::-1], np.array([], dtype=np.int64), np.array([40])]
    got = sf.decode(cols)
    for c, g in zip(cols, got):
        assert g.shape == (ns, c.size)
        assert np.array_equal(g.view(np.uint32), want[:, c].view(np.uint32))


def test_shot_roundtrip(tmp_path):
    from ertm_b200 import segy
    shot = _make_shot(120.0)
    path = tmp_path / "shot.sgy"
    segy.write_segy_shot(shot, path)
    loaded = segy.read_segy_shots(path)
    assert len(loaded) == 1
    r = loaded[0]
    assert r.receivers.nrec == shot.receivers.nrec and r.dt == pytest.approx(shot.dt, abs=1e-9)
    assert r.source.x == pytest.approx(shot.source.x, abs=1e-3)
    assert np.array_equal(r.data, shot.data)           # IEEE: exact
    assert np.allclose(r.receivers.x, shot.receivers.x, atol=1e-6)
    assert r.meta["input"] == "segy" and r.meta["group_key"] == "0" and r.components["p"] is r.data
    segy.write_segy_shot(shot, tmp_path / "ibm.sgy", fmt=1)
    ibm = segy.read_segy_shots(tmp_path / "ibm.sgy")[0]
    assert np.allclose(ibm.data, shot.data, atol=2e-3)
    assert np.array_equal(ibm.data, orc.ibm_to_float32(orc.float32_to_ibm(shot.data)))


def test_multi_shot_grouping(tmp_path):
    from ertm_b200 import segy
    shots = [_make_shot(100.0), _make_shot(300.0)]
    path = tmp_path / "multi.sgy"
    segy.write_segy_shots(shots, path)
    grouped = segy.read_segy_shots(path, segy.SegYReadOptions(group_by="source"))
    single = segy.read_segy_shots(path, segy.SegYReadOptions(group_by="file"))
    by_field = segy.read_segy_shots(path, segy.SegYReadOptions(group_by="field_record", shot_limit=1))
    assert len(grouped) == 2 and len(single) == 1 and len(by_field) == 1
    assert single[0].receivers.nrec == 22
    assert sorted(r.source.x for r in grouped) == [100.0, 300.0]
    for r, s in zip(sorted(grouped, key=lambda r: r.source.x), shots):
        assert np.array_equal(r.data, s.data)
    assert np.array_equal(by_field[0].data, shots[0].data)


def test_offset_sort_and_depth_from_group_y(tmp_path):
    from ertm_b200 import segy
    from ertm_b200.types import ReceiverSpec
    shot = _make_shot(50.0, nrec=9)
    perm = np.array([4, 0, 8, 2, 6, 1, 3, 7, 5])
    shot.receivers = ReceiverSpec(x=shot.receivers.x[perm], z=np.arange(9) * 5.0 + 10.0, component="p")
    segy.write_segy_shot(shot, tmp_path / "p.sgy")
    r = segy.read_segy_shots(tmp_path / "p.sgy", segy.SegYReadOptions(receiver_depth_from="group_y"))[0]
    order = np.argsort(shot.receivers.x)
    assert np.array_equal(r.data, shot.data[:, order])
    assert np.array_equal(r.receivers.z, shot.receivers.z[order])
    r2 = segy.read_segy_shots(tmp_path / "p.sgy", segy.SegYReadOptions(sort_by_offset=False))[0]
    assert np.array_equal(r2.data, shot.data)


def test_directory_glob_and_components(tmp_path):
    from ertm_b200 import segy
    shots = [_make_shot(100.0, nrec=5), _make_shot(200.0, nrec=5)]
    d = tmp_path / "line1"
    d.mkdir()
    segy.write_segy_shot(shots[0], d / "shot_001.sgy")
    segy.write_segy_shot(shots[1], d / "shot_002.sgy")
    by_dir = segy.read_segy_shots(d)
    by_glob = segy.read_segy_shots(str(d / "*.sgy"))
    assert len(by_dir) == 2 and len(by_glob) == 2
    assert sorted(round(float(r.source.x)) for r in by_dir) == [100, 200]
    s = segy.summarize_segy(d)
    assert (s["n_files"], s["n_shots"], s["n_traces"]) == (2, 2, 10)
    merged = segy.read_segy_components({"p": d / "shot_001.sgy", "vz": d / "shot_002.sgy"})
    assert len(merged) == 1 and list(merged[0].components) == ["p", "vz"]
    assert np.array_equal(merged[0].data, shots[0].data)
    assert np.array_equal(merged[0].components["vz"], shots[1].data)


def test_image_roundtrip(tmp_path):
    from ertm_b200 import segy
    from ertm_b200.types import GridSpec, ImageResult
    grid = GridSpec(nx=13, nz=17, dx=10.0, dz=5.0)
    image = ImageResult(image=np.random.default_rng(3).normal(size=grid.shape).astype(np.float32), grid=grid,
                        mode="pp")
    path = tmp_path / "image.sgy"
    segy.write_segy_image(image, path)
    back, dz, x = segy.read_segy_image(path)
    assert back.shape == grid.shape and dz == pytest.approx(grid.dz, abs=1e-6)
    assert np.allclose(x, np.arange(grid.nx) * grid.dx, atol=1e-6)
    assert np.array_equal(back, image.image)


def test_extended_headers_single_trace_and_limits(tmp_path):
    """A file with one extended textual header and a single trace; a shot limit."""
    from ertm_b200 import segy
    rec = np.arange(37, dtype=np.float32)[:, None] * 0.5 - 3.0
    blob = bytearray(orc.segy_bytes(rec, [{"SourceX": 7, "GroupX": 9, "TRACE_SAMPLE_COUNT": 37}], 250, 1, "x"))
    blob[3504:3506] = (1).to_bytes(2, "big")            # one extended textual header follows the binary header
    blob[3600:3600] = b"\x40" * 3200
    p = tmp_path / "ext.sgy"
    p.write_bytes(bytes(blob))
    (s,) = segy.read_segy_shots(p)
    assert s.data.shape == (37, 1) and s.dt == pytest.approx(2.5e-4)
    assert np.array_equal(s.data, orc.ibm_to_float32(orc.float32_to_ibm(rec)))
    assert s.source.x == 7.0 and s.receivers.x.tolist() == [9.0]
    shots = [_make_shot(100.0 + 50 * k, nrec=3, nt=20) for k in range(4)]
    segy.write_segy_shots(shots, tmp_path / "four.sgy")
    two = segy.read_segy_shots(tmp_path / "four.sgy", segy.SegYReadOptions(shot_limit=2))
    assert [r.source.x for r in two] == [100.0, 150.0]
    for r, s0 in zip(two, shots):
        assert np.array_equal(r.data, s0.data)


def test_decode_rejects_columns_outside_the_file_or_output():
    import ctypes as C
    from ertm_b200 import _lib
    L = _lib.lib()
    ns, ntr = 8, 3
    section = np.zeros(ntr * (240 + 4 * ns), dtype=np.uint8)
    out = np.zeros(ns * ntr, dtype=np.float32)

    def call(order, dest, width, fmt=5, out_len=out.size):
        o = np.asarray(order, dtype=np.int32)
        d = np.asarray(dest, dtype=np.int64)
        w = np.asarray(width, dtype=np.int32)
        return L.ertm_segy_decode(section.ctypes.data, ntr, ns, fmt, o.size, o.ctypes.data, d.ctypes.data,
                                  w.ctypes.data, out.ctypes.data, out_len, None)
    assert call([0, 1, 2], [0, 1, 2], [3, 3, 3]) == 0
    assert call([0, 3], [0, 1], [3, 3]) != 0                 # trace 3 of 3
    assert call([0, -1], [0, 1], [3, 3]) != 0
    assert call([0, 1], [0, 22], [3, 3]) != 0                # 22 + 7·3 beyond 24 floats
    assert call([0], [0], [0]) != 0
    assert call([0], [0], [1], fmt=3) != 0
    assert "outside" in _lib.last_error() or "format" in _lib.last_error()
    bad = C.c_int32(0)
    assert L.ertm_segy_encode(None, 1, 1, 5, C.addressof(bad), C.addressof(bad), None) != 0
