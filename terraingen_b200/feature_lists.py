"""Crater and boulder lists as the reference writes them (WriteCraterList and WriteBoulderList,
src/io/feature_lists.cpp:395-423).

The columns come straight from the arrays a population hands over (tg_crater_generate's x, y,
diameter, age and id; a boulder layer's placed boulders), host arrays or CUDA tensors. CSV has a
header row, doubles as `%.17g`, an unknown value empty, ids and integers in decimal and the flags
as 1 or 0 (CsvText, feature_lists.cpp:84-95). JSON is an object {"craters": [...]} (or
"boulders") of one object per row keyed by column in order, indented by 2 (nlohmann's
ordered_json dumped with indent 2): doubles in the shortest form that reads back exactly, NaN,
infinities and unknown values as null. The format follows the path's extension (".json" is JSON,
anything else CSV: InferListFormat, feature_lists.cpp:27).
"""

from __future__ import annotations

import math
from pathlib import Path

import numpy as np

CRATER_COLUMNS = ("x", "y", "diameter", "age_gyr", "id", "manual", "replace")

# kBoulderColumns (feature_lists.cpp:65-82), in the file's order.
BOULDER_COLUMNS = ("x", "y", "ground", "diameter", "height", "burial", "yaw_deg", "lean_deg",
                   "id", "model", "wear", "parent", "piece", "rest", "tilt_deg",
                   "tilt_azimuth_deg")

RADIAN = 180.0 / math.pi  # kRadian (include/terraingen/geometry/geometry.h:18)


def _host(values, dtype) -> np.ndarray:
    if hasattr(values, "detach"):
        values = values.detach().cpu().numpy()
    return np.ascontiguousarray(values, dtype)


def _csv_double(v: float) -> str:
    # FormatNumber(value, 17) is printf's %.17g: glibc writes a NaN's sign.
    if math.isnan(v):
        return "-nan" if math.copysign(1.0, v) < 0 else "nan"
    return "%.17g" % v


def _json_double(v: float) -> str:
    """A double as nlohmann's dump writes it: the shortest digits that read back (Python's repr
    finds the same ones), fixed notation while the decimal point falls within 15 digits left of
    the first digit or 3 zeros right of it, else d.ddde+XX; NaN and infinities as null."""
    if not math.isfinite(v):
        return "null"
    text = repr(v)
    if 1e15 <= abs(v) < 1e16:
        # repr stays fixed up to 16 integer digits where nlohmann changes to an exponent.
        sign = "-" if v < 0 else ""
        digits = text.lstrip("-").replace(".", "").rstrip("0")
        mantissa = digits[0] + ("." + digits[1:] if len(digits) > 1 else "")
        return f"{sign}{mantissa}e+15"
    return text


def _dump(path: Path, key: str, names, rows) -> None:
    """Writes {key: [rows]} as nlohmann's dump(2) lays it out; each row holds JSON texts."""
    if not rows:
        path.write_text('{\n  "%s": []\n}\n' % key)
        return
    out = ['{\n  "%s": [\n' % key]
    for r, row in enumerate(rows):
        cells = ",\n".join(f'      "{name}": {value}' for name, value in zip(names, row))
        out.append("    {\n" + cells + "\n    }" + (",\n" if r + 1 < len(rows) else "\n"))
    out.append("  ]\n}\n")
    path.write_text("".join(out))


def _format(path: Path, format: str | None) -> str:
    fmt = format or ("json" if path.suffix.lower() == ".json" else "csv")
    if fmt not in ("csv", "json"):
        raise ValueError("format must be csv or json")
    return fmt


def write_crater_list(path, x, y, diameter, age_gyr, ids, manual=None, replace=None,
                      format: str | None = None) -> None:
    """Writes the craters to `path`; `format` "csv" or "json" overrides the extension."""
    cols = [_host(v, np.float64) for v in (x, y, diameter, age_gyr)]
    n = len(cols[0])
    ident = _host(ids, np.uint64)
    man = np.zeros(n, bool) if manual is None else _host(manual, bool)
    rep = np.zeros(n, bool) if replace is None else _host(replace, bool)
    if any(len(c) != n for c in (*cols, ident, man, rep)):
        raise ValueError("every column needs one value per crater")
    path = Path(path)
    if _format(path, format) == "csv":
        lines = [",".join(CRATER_COLUMNS)]
        for i in range(n):
            cells = [_csv_double(float(c[i])) for c in cols]
            cells += [str(int(ident[i])), "1" if man[i] else "0", "1" if rep[i] else "0"]
            lines.append(",".join(cells))
        path.write_text("\n".join(lines) + "\n")
        return
    rows = []
    for i in range(n):
        row = [_json_double(float(c[i])) for c in cols]
        row += [str(int(ident[i])), "true" if man[i] else "false", "true" if rep[i] else "false"]
        rows.append(row)
    _dump(path, "craters", CRATER_COLUMNS, rows)


def write_boulder_list(path, x, y, diameter, height, burial=None, yaw=None, lean=None, ids=None,
                       ground=None, model=None, wear=None, parent=None, piece=None, rest=None,
                       tilt=None, tilt_azimuth=None, format: str | None = None) -> None:
    """Writes the boulders to `path` (WriteBoulderList, feature_lists.cpp:412-423); `format`
    "csv" or "json" overrides the extension.

    Each argument is one value per boulder, as the reference's Boulder holds it
    (include/terraingen/layers/boulders/boulder.h:52-80): yaw, lean, tilt and tilt_azimuth in
    radians (written in degrees), rest 0 Face, 1 Side or 2 End, model a flag, parent and piece
    the fragment's origin. `ground` is the height beneath the center where the layer knows it:
    NaN (or no array) writes it as unknown. Columns left out are the reference's defaults (0,
    unknown ground, a whole boulder resting on its face)."""
    x = _host(x, np.float64)
    n = len(x)

    def col(values, dtype, fill=0):
        return np.full(n, fill, dtype) if values is None else _host(values, dtype)

    doubles = {"x": x, "y": _host(y, np.float64), "diameter": _host(diameter, np.float64),
               "height": _host(height, np.float64), "burial": col(burial, np.float64),
               "wear": col(wear, np.float64), "ground": col(ground, np.float64, np.nan)}
    for name, values in (("yaw_deg", yaw), ("lean_deg", lean), ("tilt_deg", tilt),
                         ("tilt_azimuth_deg", tilt_azimuth)):
        doubles[name] = col(values, np.float64) * RADIAN
    ints = {"id": col(ids, np.uint64), "parent": col(parent, np.uint64),
            "piece": col(piece, np.uint32).astype(np.uint64), "rest": col(rest, np.int64)}
    flags = col(model, bool)
    if any(len(c) != n for c in (*doubles.values(), *ints.values(), flags)):
        raise ValueError("every column needs one value per boulder")
    path = Path(path)
    fmt = _format(path, format)
    cells = []
    for name in BOULDER_COLUMNS:
        if name == "model":
            on, off = ("1", "0") if fmt == "csv" else ("true", "false")
            cells.append([on if f else off for f in flags])
        elif name in ints:
            cells.append([str(int(v)) for v in ints[name]])
        elif name == "ground":
            # An unknown ground (std::optional without a value) is empty in CSV, null in JSON.
            known = ~np.isnan(doubles[name])
            text = _csv_double if fmt == "csv" else _json_double
            empty = "" if fmt == "csv" else "null"
            cells.append([text(float(v)) if k else empty for v, k in zip(doubles[name], known)])
        else:
            text = _csv_double if fmt == "csv" else _json_double
            cells.append([text(float(v)) for v in doubles[name]])
    rows = [list(r) for r in zip(*cells)] if n else []
    if fmt == "csv":
        lines = [",".join(BOULDER_COLUMNS)] + [",".join(r) for r in rows]
        path.write_text("\n".join(lines) + "\n")
    else:
        _dump(path, "boulders", BOULDER_COLUMNS, rows)
