"""Wire formats on the host: the .npz store against files the reference's own
NumpyDataStore wrote (tests/golden/store/, data.py:73-297), the IBM float
definition's known answers, and SEG-Y header handling on files the oracle
builds (the sample codec itself runs on the GPU: tests/test_gpu_formats.py)."""

from __future__ import annotations

import json

import numpy as np
import pytest

from helpers import GOLDEN, load
from oracle import ertm_oracle as orc
from ertm_b200 import segy
from ertm_b200.data import NumpyDataStore
from ertm_b200.exceptions import DataError
from ertm_b200.types import ElasticModel, GridSpec

STORE = GOLDEN / "store"


def _npz(path):
    with np.load(path, allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


def test_loads_reference_written_files():
    fx = load("store")
    st = NumpyDataStore.__new__(NumpyDataStore)
    m = st.load_model(STORE / "model.npz")
    assert (m.grid.nx, m.grid.nz, m.grid.dx, m.grid.dz) == (19, 13, 10.0, 10.0)
    assert m.name == "store-model" and m.meta == {"builder": "layered", "layers": 3}
    for k in ("vp", "vs", "rho", "qp", "qs"):
        assert np.array_equal(getattr(m, k), fx[k]) and getattr(m, k).dtype == np.float32
    s = st.load_shot(STORE / "shot.npz")
    assert s.dt == 5e-4 and s.receivers.component == "p" and s.meta == {"synthetic": True, "engine": "elastic"}
    assert (s.source.x, s.source.z, s.source.f0, s.source.amplitude, s.source.delay, s.source.mechanism) == \
        (90.0, 20.0, 25.0, 2.0, 0.01, "shear")
    assert list(s.components) == ["p", "vx", "vz"]
    for k in ("p", "vx", "vz"):
        assert np.array_equal(s.components[k], fx[f"comp_{k}"])
    assert np.array_equal(s.data, fx["data"]) and np.array_equal(s.t, fx["t"])
    assert np.array_equal(s.receivers.x, fx["rx"]) and np.array_equal(s.receivers.z, fx["rz"])
    im = st.load_image(STORE / "image.npz")
    assert im.mode == "ps" and im.meta == {"condition": "normalized", "n_shots": 3}
    assert np.array_equal(im.image, fx["image"])


@pytest.mark.parametrize("kind", ["model", "shot", "image"])
def test_written_files_match_reference_written(tmp_path, kind):
    st = NumpyDataStore(tmp_path)
    obj = getattr(st, f"load_{kind}")(STORE / f"{kind}.npz")
    path = getattr(st, f"save_{kind}")(obj, kind)
    assert path == tmp_path / f"{kind}s" / f"{kind}.npz"
    ours, ref = _npz(path), _npz(STORE / f"{kind}.npz")
    assert list(ours) == list(ref)
    for k in ref:
        assert ours[k].dtype == ref[k].dtype and ours[k].shape == ref[k].shape, k
        assert np.array_equal(ours[k], ref[k]), k
    assert str(ours["meta"]) == str(ref["meta"])          # same JSON text, key order included
    assert sorted(p.name for p in tmp_path.iterdir()) == ["images", "logs", "models", "reports", "shots"]


def test_store_errors(tmp_path):
    st = NumpyDataStore(tmp_path)
    bad = tmp_path / "bad.npz"
    np.savez(bad, vp=np.ones((2, 2)), meta=np.array("[1, 2]"))
    with pytest.raises(DataError):
        st.load_model(bad)
    with pytest.raises(DataError):
        st.load_image(tmp_path / "missing.npz")
    g = GridSpec(nx=3, nz=2, dx=1.0, dz=1.0)
    one = np.ones(g.shape, np.float32)
    m = ElasticModel(grid=g, vp=one, vs=one * 2, rho=one, qp=one, qs=one)     # vs >= vp
    np.savez(tmp_path / "m.npz", vp=m.vp, vs=m.vs, rho=m.rho, qp=m.qp, qs=m.qs,
             meta=np.array(json.dumps({"grid": {"nx": 3, "nz": 2, "dx": 1.0, "dz": 1.0}})))
    with pytest.raises(DataError):
        st.load_model(tmp_path / "m.npz")
    with pytest.raises(DataError):
        st.save_json({"a": 1}, "x", subdir="nope")
    assert json.loads(st.save_json({"a": 1}, "x").read_text()) == {"a": 1}


# ---------------------------------------------------------------------------
# IBM hexadecimal float: known answers from the format's definition
# ---------------------------------------------------------------------------
IBM_KNOWN = [(1.0, 0x41100000), (-118.625, 0xC276A000), (0.15625, 0x40280000), (0.03125, 0x3F800000),
             (0.0, 0x00000000), (-1.0, 0xC1100000), (16.0, 0x42100000), (0.5, 0x40800000)]


def test_ibm_known_answers():
    for v, w in IBM_KNOWN:
        assert int(orc.float32_to_ibm(np.float32(v))) == w
        assert float(orc.ibm_to_float32(w)) == v
    big = orc.ibm_to_float32([0x7FFFFFFF, 0xFFFFFFFF, 0x00100000])
    assert np.isposinf(big[0]) and np.isneginf(big[1]) and big[2] == 0.0
    assert int(orc.float32_to_ibm(np.float32(np.inf))) == 0x7FFFFFFF


def test_ibm_round_trip_within_format_precision():
    bits = np.random.default_rng(0).integers(0, 2 ** 32, 4000, dtype=np.uint64).astype(np.uint32)
    x = bits.view(np.float32)
    x = x[np.isfinite(x)]
    back = orc.ibm_to_float32(orc.float32_to_ibm(x)).astype(np.float64)
    rel = np.abs(back - x) / np.maximum(np.abs(x.astype(np.float64)), np.finfo(np.float64).tiny)
    assert rel.max() <= 2.0 ** -21                       # half a unit of a 21-bit fraction
    ints = np.arange(-(1 << 20), 1 << 20, 997, dtype=np.float32)      # 21 significant bits: exact
    assert np.array_equal(orc.ibm_to_float32(orc.float32_to_ibm(ints)), ints)


# ---------------------------------------------------------------------------
# SEG-Y headers on oracle-built files (no sample decoding)
# ---------------------------------------------------------------------------
def _shot_file(path, sx, nrec=5, ns=64, fmt=5, scalar=1, field=1):
    rng = np.random.default_rng(int(sx))
    rec = rng.normal(size=(ns, nrec)).astype(np.float32)
    gx = np.linspace(0.0, 200.0, nrec)
    heads = [{"SourceX": round(sx * (abs(scalar) if scalar < 0 else 1)), "SourceY": 20,
              "GroupX": round(g * (abs(scalar) if scalar < 0 else 1)), "GroupY": 20, "SourceGroupScalar": scalar,
              "offset": round(abs(g - sx)), "FieldRecord": field, "TraceNumber": k + 1,
              "TRACE_SAMPLE_COUNT": ns, "TRACE_SAMPLE_INTERVAL": 400} for k, g in enumerate(gx)]
    path.write_bytes(orc.segy_bytes(rec, heads, 400, fmt, f"shot {sx}"))
    return rec, heads


def test_open_segy_headers_match_oracle(tmp_path):
    p = tmp_path / "a.sgy"
    _, heads = _shot_file(p, 120.0, scalar=-10)
    sf = segy.open_segy(p)
    assert (sf.ns, sf.fmt, sf.interval, sf.n_traces) == (64, 5, 400, 5)
    binh, oheads, _ = orc.segy_parse(p.read_bytes())
    for name in segy.TRACE_FIELDS:
        assert sf.headers[name].tolist() == [h[name] for h in oheads], name
    assert np.allclose(segy.apply_scalar(sf.headers["GroupX"], sf.headers["SourceGroupScalar"]),
                       np.linspace(0.0, 200.0, 5))


def test_summary_directory_and_glob(tmp_path):
    d = tmp_path / "line1"
    d.mkdir()
    _shot_file(d / "shot_001.sgy", 100.0)
    _shot_file(d / "shot_002.sgy", 200.0)
    (d / "notes.txt").write_text("x")
    s = segy.summarize_segy(d)
    assert (s["n_files"], s["n_shots"], s["n_traces"], s["ns"]) == (2, 2, 10, 64)
    assert s["dt"] == pytest.approx(4e-4) and s["source_x_range"] == [100.0, 200.0]
    assert s["offset_range"] == [0.0, 200.0]
    assert [p.name for p in segy.expand_segy_paths(str(d / "*.sgy"))] == ["shot_001.sgy", "shot_002.sgy"]
    with pytest.raises(DataError):
        segy.expand_segy_paths(str(d / "*.segy"))
    with pytest.raises(DataError):
        segy.expand_segy_paths(tmp_path / "missing.sgy")


def test_open_segy_rejects_bad_files(tmp_path):
    p = tmp_path / "a.sgy"
    _shot_file(p, 50.0)
    blob = p.read_bytes()
    (tmp_path / "cut.sgy").write_bytes(blob[:-7])
    with pytest.raises(DataError):
        segy.open_segy(tmp_path / "cut.sgy")
    (tmp_path / "tiny.sgy").write_bytes(blob[:100])
    with pytest.raises(DataError):
        segy.open_segy(tmp_path / "tiny.sgy")
    bad = bytearray(blob)
    bad[3224:3226] = (3).to_bytes(2, "big")             # format 3 (int16) is not supported
    (tmp_path / "fmt.sgy").write_bytes(bytes(bad))
    with pytest.raises(DataError):
        segy.open_segy(tmp_path / "fmt.sgy")
    with pytest.raises(DataError):
        segy.SegYReadOptions(group_by="line").validate()


def test_apply_scalar():
    v = np.array([100, 100, 100, 100])
    assert segy.apply_scalar(v, np.array([0, 10, -10, 1])).tolist() == [100.0, 1000.0, 10.0, 100.0]
