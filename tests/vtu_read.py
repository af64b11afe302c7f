"""Reader for the VTK XML unstructured-grid files that LSSolver::solve
writes (inline binary arrays: base64 of a 64-bit byte count and the values).
Test infrastructure."""
import base64
import xml.etree.ElementTree as ET

import numpy as np

_TYPES = {"Float32": np.float32, "Float64": np.float64, "Int32": np.int32, "UInt8": np.uint8}


def _array(e):
    dt = _TYPES[e.get("type")]
    comps = int(e.get("NumberOfComponents", "1"))
    text = (e.text or "").strip()
    if e.get("format") == "binary":
        raw = base64.b64decode(text) if text else b""
        n = int(np.frombuffer(raw[:8], np.uint64)[0]) if raw else 0
        a = np.frombuffer(raw[8:8 + n], dt)
    else:
        a = np.array(text.split(), dt) if text else np.zeros(0, dt)
    return a.reshape(-1, comps) if comps > 1 else a


def read(path):
    """Points, cells (connectivity, offsets, types), point data and the
    TIME / STEP field data of one file."""
    root = ET.parse(path).getroot()
    grid = root.find("UnstructuredGrid")
    out = {"field": {}, "point_data": {}}
    for e in grid.find("FieldData"):
        out["field"][e.get("Name")] = _array(e)[0]
    piece = grid.find("Piece")
    out["n_points"] = int(piece.get("NumberOfPoints"))
    out["n_cells"] = int(piece.get("NumberOfCells"))
    out["points"] = _array(piece.find("Points").find("DataArray")).reshape(-1, 3)
    for e in piece.find("Cells"):
        out[e.get("Name")] = _array(e)
    for e in piece.find("PointData"):
        out["point_data"][e.get("Name")] = _array(e)
    return out
