"""SEG-Y input and output with the trace samples coded on the device (segy.py
of the reference, which reads and writes through segyio 1.9.15).

The file layout is SEG-Y revision 1: a 3200-byte textual header (EBCDIC),
a 400-byte binary header, optional 3200-byte extended textual headers, then
fixed-length trace blocks of a 240-byte trace header and ``ns`` big-endian
4-byte samples (data sample format 5, IEEE single, or 1, IBM hexadecimal
single).  Headers are parsed on the host as NumPy structured views, with no
per-trace Python loop; the samples of every shot of a file are decoded in one
``ertm_segy_decode`` launch that converts and transposes them straight into
``(nt, nrec)`` records in grouped, offset-sorted order, and writing runs the
inverse ``ertm_segy_encode``.  Field positions follow the standard; the
reference addresses the same fields through segyio's ``BinField`` /
``TraceField`` names, which are the names used here.
"""

from __future__ import annotations

import glob as _glob
from dataclasses import dataclass
from pathlib import Path
from typing import Any, Sequence

import numpy as np

from . import _lib
from .exceptions import DataError
from .types import ImageResult, ReceiverSpec, ShotRecord, SourceSpec

TEXT_BYTES, BINARY_BYTES, TRACE_HEADER_BYTES = 3200, 400, 240
SAMPLE_FORMATS = (1, 5)

# binary header fields: name -> (byte offset inside the 400-byte block, type)
BIN_FIELDS = {
    "Interval": (16, ">u2"), "Samples": (20, ">u2"), "Format": (24, ">i2"), "Sorting": (28, ">i2"),
    "SEGYRevision": (300, ">u2"), "TraceFlag": (302, ">i2"), "ExtendedHeaders": (304, ">i2"),
}
# trace header fields: name -> (byte offset inside the 240-byte header, type)
TRACE_FIELDS = {
    "FieldRecord": (8, ">i4"), "TraceNumber": (12, ">i4"), "CDP": (20, ">i4"), "offset": (36, ">i4"),
    "SourceGroupScalar": (70, ">i2"), "SourceX": (72, ">i4"), "SourceY": (76, ">i4"), "GroupX": (80, ">i4"),
    "GroupY": (84, ">i4"), "TRACE_SAMPLE_COUNT": (114, ">u2"), "TRACE_SAMPLE_INTERVAL": (116, ">u2"),
}


def _struct(fields: dict[str, tuple[int, str]], size: int) -> np.dtype:
    return np.dtype({"names": list(fields), "formats": [t for _, t in fields.values()],
                     "offsets": [o for o, _ in fields.values()], "itemsize": size})


BIN_DTYPE = _struct(BIN_FIELDS, BINARY_BYTES)
TRACE_DTYPE = _struct(TRACE_FIELDS, TRACE_HEADER_BYTES)


@dataclass(frozen=True)
class SegYReadOptions:
    """Read options (segy.py:63-86)."""

    component: str = "p"
    group_by: str = "source"            # source | field_record | file
    receiver_depth: float = 0.0
    source_depth: float = 0.0
    receiver_depth_from: str = "constant"  # constant | group_y
    coordinate_scalar: int | None = None
    shot_limit: int = 0
    sort_by_offset: bool = True
    f0: float = 20.0
    delay: float = 0.0

    def validate(self) -> None:
        if self.group_by not in {"source", "field_record", "file"}:
            raise DataError(f"group_by must be source/field_record/file, got {self.group_by!r}")
        if self.receiver_depth_from not in {"constant", "group_y"}:
            raise DataError(f"receiver_depth_from must be constant/group_y, got {self.receiver_depth_from!r}")
        if self.shot_limit < 0:
            raise DataError("shot_limit must not be negative")


def apply_scalar(values: np.ndarray, scalar) -> np.ndarray:
    """SEG-Y coordinate scalar: positive multiplies, negative divides, 0 leaves (segy.py:89-93)."""
    v = np.asarray(values, dtype=np.float64)
    s = np.broadcast_to(np.asarray(scalar, dtype=np.int64), v.shape)
    a = np.abs(s).astype(np.float64)
    return np.where(s < 0, v / np.where(a == 0, 1.0, a), np.where(s > 0, v * a, v))


# ----------------------------------------------------------------------------
# the file image
# ----------------------------------------------------------------------------
@dataclass
class SegYFile:
    """A SEG-Y file in host memory: binary header values, trace header view and
    the trace section (``n_traces`` blocks of ``240 + 4·ns`` bytes)."""

    path: Path
    raw: np.ndarray
    interval: int
    ns: int
    fmt: int
    first_trace: int
    n_traces: int

    @property
    def trace_bytes(self) -> int:
        return TRACE_HEADER_BYTES + 4 * self.ns

    @property
    def headers(self) -> np.ndarray:
        return np.ndarray((self.n_traces,), dtype=TRACE_DTYPE, buffer=self.raw, offset=self.first_trace,
                          strides=(self.trace_bytes,))

    def section_ptr(self) -> int:
        return self.raw.ctypes.data + self.first_trace

    def decode(self, columns: Sequence[np.ndarray]) -> list[np.ndarray]:
        """float32 records ``(ns, len(c))``, one per column list of trace indices."""
        widths = [int(np.asarray(c).size) for c in columns]
        total = self.ns * sum(widths)
        out = np.empty(max(total, 1), dtype=np.float32)
        if total:
            order = np.ascontiguousarray(np.concatenate([np.asarray(c, dtype=np.int64) for c in columns]),
                                         dtype=np.int32)
            base = np.cumsum([0] + [self.ns * w for w in widths[:-1]])
            dest = np.ascontiguousarray(np.concatenate([b + np.arange(w) for b, w in zip(base, widths)]),
                                        dtype=np.int64)
            width = np.ascontiguousarray(np.repeat(np.asarray(widths, dtype=np.int32), widths))
            _lib.check(_lib.lib().ertm_segy_decode(self.section_ptr(), self.n_traces, self.ns, self.fmt,
                                                  order.size, _lib.ptr(order), _lib.ptr(dest), _lib.ptr(width),
                                                  _lib.ptr(out), out.size, None), "segy decode")
        recs, pos = [], 0
        for w in widths:
            recs.append(out[pos:pos + self.ns * w].reshape(self.ns, w))
            pos += self.ns * w
        return recs


def open_segy(path: str | Path) -> SegYFile:
    """Read a SEG-Y file's bytes and headers (no sample decoding)."""
    p = Path(path)
    try:
        raw = np.fromfile(p, dtype=np.uint8)
    except OSError as exc:
        raise DataError(f"cannot read SEG-Y: {p}: {exc}") from exc
    if raw.size < TEXT_BYTES + BINARY_BYTES:
        raise DataError(f"not a SEG-Y file (only {raw.size} bytes): {p}")
    b = np.ndarray((), dtype=BIN_DTYPE, buffer=raw, offset=TEXT_BYTES)
    ns, fmt, n_ext = int(b["Samples"]), int(b["Format"]), max(int(b["ExtendedHeaders"]), 0)
    interval = int(b["Interval"]) or 1000
    if fmt not in SAMPLE_FORMATS:
        raise DataError(f"SEG-Y data sample format {fmt} is not supported (1 IBM float, 5 IEEE float): {p}")
    if ns < 1:
        raise DataError(f"SEG-Y binary header gives {ns} samples per trace: {p}")
    first = TEXT_BYTES + BINARY_BYTES + TEXT_BYTES * n_ext
    tb = TRACE_HEADER_BYTES + 4 * ns
    body = raw.size - first
    if body < 0 or body % tb:
        raise DataError(f"SEG-Y trace section of {body} bytes is not whole traces of {tb} bytes: {p}")
    return SegYFile(path=p, raw=raw, interval=interval, ns=ns, fmt=fmt, first_trace=first, n_traces=body // tb)


def expand_segy_paths(path: str | Path) -> list[Path]:
    """A file, a directory of .sgy/.segy files, or a wildcard pattern → sorted files (segy.py:158-185)."""
    text = str(path)
    if any(ch in text for ch in "*?["):
        files = [p for p in sorted(Path(m) for m in _glob.glob(text)) if p.is_file()]
        if not files:
            raise DataError(f"no SEG-Y file matches {text}")
        return files
    cand = Path(text)
    if cand.is_dir():
        files = sorted(p for p in cand.iterdir() if p.is_file() and p.suffix.lower() in {".sgy", ".segy"})
        if not files:
            raise DataError(f"no SEG-Y file in directory {cand}")
        return files
    if not cand.is_file():
        raise DataError(f"SEG-Y file does not exist: {cand}")
    return [cand]


def summarize_segy(path: str | Path) -> dict[str, Any]:
    """Header-only summary of one or many files (segy.py:188-234)."""
    files = expand_segy_paths(path)
    n_traces = n_shots = 0
    dts, nss = set(), set()
    sx_all, gx_all, off_all = [], [], []
    for f in files:
        sf = open_segy(f)
        h = sf.headers
        sx = apply_scalar(h["SourceX"], h["SourceGroupScalar"])
        gx = apply_scalar(h["GroupX"], h["SourceGroupScalar"])
        sx_all.append(sx)
        gx_all.append(gx)
        off_all.append(np.abs(h["offset"].astype(np.int64)).astype(np.float64))
        n_traces += sf.n_traces
        n_shots += len(set(sx.tolist()))
        dts.add(sf.interval * 1e-6)
        nss.add(sf.ns)
    cat = lambda parts: np.concatenate(parts) if parts else np.zeros(0)  # noqa: E731
    sx, gx, off = cat(sx_all), cat(gx_all), cat(off_all)
    rng = lambda a: [float(a.min()), float(a.max())] if a.size else [float("inf"), float("-inf")]  # noqa: E731
    return {"files": [str(f) for f in files], "n_files": len(files), "n_traces": int(n_traces),
            "n_shots": int(n_shots), "dt": sorted(dts)[0] if len(dts) == 1 else sorted(dts),
            "ns": sorted(nss)[0] if len(nss) == 1 else sorted(nss), "source_x_range": rng(sx),
            "receiver_x_range": rng(gx), "offset_range": rng(off)}


def _read_single(path: Path, opts: SegYReadOptions) -> list[ShotRecord]:
    """One file → its shots (segy.py:255-320)."""
    sf = open_segy(path)
    h = sf.headers
    scalar = opts.coordinate_scalar or h["SourceGroupScalar"]
    sources = apply_scalar(h["SourceX"], scalar)
    groups = apply_scalar(h["GroupX"], scalar)
    group_y = apply_scalar(h["GroupY"], scalar)
    if opts.group_by == "file":
        keys = np.zeros(sf.n_traces, dtype=np.int64)
    elif opts.group_by == "field_record":
        keys = h["FieldRecord"].astype(np.int64)
    else:
        keys = np.unique(sources, return_inverse=True)[1]
    dt = sf.interval * 1e-6
    columns, uniq = [], np.unique(keys)
    for key in uniq:
        index = np.where(keys == key)[0]
        if opts.sort_by_offset:
            index = index[np.argsort(groups[index])]
        columns.append(index)
    if opts.shot_limit:
        columns, uniq = columns[:int(opts.shot_limit)], uniq[:int(opts.shot_limit)]
    records = sf.decode(columns)
    shots = []
    for key, index, rec in zip(uniq, columns, records):
        rz = group_y[index] if opts.receiver_depth_from == "group_y" else np.full(index.size,
                                                                                   float(opts.receiver_depth))
        shot = ShotRecord(
            data=rec, dt=dt, t=np.arange(rec.shape[0], dtype=np.float64) * dt,
            receivers=ReceiverSpec(x=groups[index], z=rz, component=opts.component),
            source=SourceSpec(x=float(sources[index[0]]), z=float(opts.source_depth), f0=float(opts.f0),
                              kind="ricker", amplitude=1.0, delay=float(opts.delay)),
            meta={"input": "segy", "file": str(path), "component": opts.component, "group_by": opts.group_by,
                  "group_key": str(key), "n_traces": int(index.size), "placeholder": False},
            components={opts.component: rec})
        shots.append(shot.validate())
    return shots


def read_segy_shots(path: str | Path, options: SegYReadOptions | None = None) -> list[ShotRecord]:
    """Shots of a file, directory or wildcard, grouped per the options (segy.py:237-252)."""
    opts = options or SegYReadOptions()
    opts.validate()
    shots: list[ShotRecord] = []
    for f in expand_segy_paths(path):
        shots.extend(_read_single(f, opts))
    return shots[:int(opts.shot_limit)] if opts.shot_limit else shots


def read_segy_components(component_files: dict[str, str | Path],
                         options: SegYReadOptions | None = None) -> list[ShotRecord]:
    """One file per component, merged shot by shot (segy.py:323-370)."""
    if not component_files:
        raise DataError("component_files must not be empty")
    base_opts = options or SegYReadOptions()
    per: dict[str, list[ShotRecord]] = {}
    for comp, path in component_files.items():
        opts = SegYReadOptions(**{**base_opts.__dict__, "component": comp})
        per[comp] = read_segy_shots(path, opts)
    counts = {k: len(v) for k, v in per.items()}
    if len(set(counts.values())) != 1:
        raise DataError(f"components hold different shot counts: {counts}")
    merged = []
    first = next(iter(per.values()))
    for i in range(len(first)):
        base = first[i]
        comps = {k: v[i].data for k, v in per.items()}
        merged.append(ShotRecord(data=comps.get("p", base.data), dt=base.dt, t=base.t, receivers=base.receivers,
                                 source=base.source, meta={**base.meta, "components": list(comps)},
                                 components=comps))
    return merged


# ----------------------------------------------------------------------------
# writing
# ----------------------------------------------------------------------------
def _rint(values) -> np.ndarray:
    """Python's round() to an integer (half to even), elementwise."""
    return np.rint(np.asarray(values, dtype=np.float64)).astype(np.int64)


def _write(path: str | Path, text: str, rec: np.ndarray, headers: np.ndarray, interval: int, fmt: int) -> Path:
    if int(fmt) not in SAMPLE_FORMATS:
        raise DataError(f"SEG-Y data sample format {fmt} is not supported (1 IBM float, 5 IEEE float)")
    target = Path(path)
    target.parent.mkdir(parents=True, exist_ok=True)
    ns, ntr = rec.shape
    if ns > 65535:
        raise DataError(f"SEG-Y rev 1 holds at most 65535 samples per trace, got {ns}")
    head = np.zeros(TEXT_BYTES + BINARY_BYTES, dtype=np.uint8)
    head[:TEXT_BYTES] = np.frombuffer(text[:TEXT_BYTES].ljust(TEXT_BYTES).encode("cp037"), dtype=np.uint8)
    b = np.ndarray((), dtype=BIN_DTYPE, buffer=head, offset=TEXT_BYTES)
    b["Interval"], b["Samples"], b["Format"], b["Sorting"] = interval, ns, int(fmt), 1
    b["SEGYRevision"], b["TraceFlag"], b["ExtendedHeaders"] = 0x0100, 1, 0
    traces = np.empty(ntr * (TRACE_HEADER_BYTES + 4 * ns), dtype=np.uint8)
    hdr = np.ascontiguousarray(headers).view(np.uint8)
    src = np.ascontiguousarray(rec, dtype=np.float32)
    _lib.check(_lib.lib().ertm_segy_encode(_lib.ptr(src), ns, ntr, int(fmt), _lib.ptr(hdr), _lib.ptr(traces), None),
               "segy encode")
    try:
        with open(target, "wb") as fh:
            fh.write(head.tobytes())
            fh.write(traces.tobytes())
    except OSError as exc:
        raise DataError(f"cannot write SEG-Y: {target}: {exc}") from exc
    return target


def _shot_headers(shots: Sequence[ShotRecord], ns: int, interval: int, *, field_from_shot: bool) -> np.ndarray:
    n = sum(int(s.data.shape[1]) for s in shots)
    h = np.zeros(n, dtype=TRACE_DTYPE)
    pos = 0
    for k, s in enumerate(shots):
        rx = np.asarray(s.receivers.x, dtype=np.float64)
        m = rx.size
        sl = slice(pos, pos + m)
        h["SourceX"][sl] = _rint(s.source.x)
        h["SourceY"][sl] = _rint(s.source.z)
        h["GroupX"][sl] = _rint(rx)
        h["GroupY"][sl] = _rint(s.receivers.z)
        h["offset"][sl] = _rint(np.abs(rx - float(s.source.x)))
        h["FieldRecord"][sl] = k + 1 if field_from_shot else 1
        pos += m
    h["SourceGroupScalar"] = 1
    h["TraceNumber"] = np.arange(1, n + 1)
    h["TRACE_SAMPLE_COUNT"] = ns
    h["TRACE_SAMPLE_INTERVAL"] = interval
    return h


def write_segy_shot(shot: ShotRecord, path: str | Path, *, fmt: int = 5, component: str | None = None) -> Path:
    """One shot, traces = receivers, samples = time (segy.py:373-423)."""
    shot.validate()
    data = np.asarray(shot.data, dtype=np.float32)
    ns = data.shape[0]
    interval = int(round(shot.dt * 1e6))
    headers = _shot_headers([shot], ns, interval, field_from_shot=False)
    return _write(path, f"ERTM shot {shot.source.x:.1f}/{shot.source.z:.1f}", data, headers, interval, fmt)


def write_segy_shots(shots: Sequence[ShotRecord], path: str | Path, *, fmt: int = 5) -> Path:
    """Many shots in one file, FieldRecord = shot number (segy.py:426-482)."""
    if not shots:
        raise DataError("writing SEG-Y needs at least one shot")
    for s in shots:
        s.validate()
    ns = int(shots[0].data.shape[0])
    if any(int(s.data.shape[0]) != ns for s in shots):
        raise DataError("every shot of one SEG-Y file needs the same record length")
    interval = int(round(shots[0].dt * 1e6))
    data = np.concatenate([np.asarray(s.data, dtype=np.float32) for s in shots], axis=1)
    headers = _shot_headers(shots, ns, interval, field_from_shot=True)
    return _write(path, f"ERTM shots x{len(shots)}", data, headers, interval, fmt)


def write_segy_image(image: ImageResult, path: str | Path, *, fmt: int = 5) -> Path:
    """Depth image, traces = x, samples = depth, Interval = dz in mm (segy.py:485-530)."""
    image.validate()
    img = np.asarray(image.image, dtype=np.float32)      # (nz, nx): samples × traces
    nz, nx = img.shape
    interval = max(int(round(float(image.grid.dz) * 1000)), 1)
    h = np.zeros(nx, dtype=TRACE_DTYPE)
    x = _rint([image.grid.x_at(i) for i in range(nx)])
    h["SourceX"], h["GroupX"], h["SourceGroupScalar"] = x, x, 1
    h["CDP"] = np.arange(1, nx + 1)
    h["TRACE_SAMPLE_COUNT"], h["TRACE_SAMPLE_INTERVAL"] = nz, interval
    return _write(path, f"ERTM image {image.mode.upper()} (depth domain)", img, h, interval, fmt)


def read_segy_image(path: str | Path) -> tuple[np.ndarray, float, np.ndarray]:
    """``(image[nz, nx], dz, x)`` of a file written by ``write_segy_image`` (segy.py:533-554)."""
    p = Path(path)
    if not p.is_file():
        raise DataError(f"SEG-Y file does not exist: {p}")
    sf = open_segy(p)
    (img,) = sf.decode([np.arange(sf.n_traces)])
    x = sf.headers["GroupX"].astype(np.float64)
    return img, sf.interval / 1000.0, x

