"""Reader for the .vti files OpenLB's SuperVTMwriter3D writes (binary,
zlib-compressed, base64: src/io/superVtmWriter3D.hh:425-500).

Each DataArray holds base64(uint32[4] {1, size, size, compressed size})
followed by base64(zlib(float32 data)), x fastest, over the piece extent
(the cuboid plus its overlap)."""
from __future__ import annotations

import base64
import re
import zlib
from pathlib import Path

import numpy as np


def read_vti(path: Path) -> dict:
    """Returns {name: array of shape (nz, ny, nx, components)} and 'extent'."""
    text = Path(path).read_text()
    m = re.search(r'<Piece Extent="([-\d ]+)"', text)
    ext = [int(v) for v in m.group(1).split()]
    shape = (ext[5] - ext[4] + 1, ext[3] - ext[2] + 1, ext[1] - ext[0] + 1)
    out = {"extent": ext}
    for arr in re.finditer(r'<DataArray type="Float32" Name="([^"]+)" NumberOfComponents="(\d+)"'
                           r'[^>]*>\s*([A-Za-z0-9+/=]+)\s*</DataArray>', text):
        name, comps, payload = arr.group(1), int(arr.group(2)), arr.group(3)
        header = np.frombuffer(base64.b64decode(payload[:24]), dtype=np.uint32)
        if header[0] != 1:
            raise ValueError(f"{path}: {name} spans {header[0]} compressed blocks")
        raw = zlib.decompress(base64.b64decode(payload[24:]))
        data = np.frombuffer(raw, dtype=np.float32)
        if data.size * 4 != header[1]:
            raise ValueError(f"{path}: {name} size mismatch")
        out[name] = data.reshape(shape + (comps,))
    return out
