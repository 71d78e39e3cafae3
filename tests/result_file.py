"""Reader of the binary map file (ResultHydro.bin): the layout swIO::initBinFileMapDecimal and
fillBinFileMapDecimal write (src/common/swIO.cpp:285-645), restated for the tests."""
import struct

import numpy as np


def geometry_prefix_length(geo: bytes) -> int:
    """Bytes of geometry.sw2d from its start to the end of the node-to-cell lists."""
    off = 0

    def u64(n=1):
        nonlocal off
        v = struct.unpack_from(f"<{n}Q", geo, off)
        off += 8 * n
        return v

    (vlen,) = u64()
    off += vlen
    nc, nb, ni, nn, nbnd = u64(5)
    links = []
    for _ in range(nc):
        cnt = u64(6)
        off += 40
        links.append(cnt[2] + cnt[3] + cnt[4] + cnt[5])
    node_cells = []
    for _ in range(nn):
        rec = struct.unpack_from("<2Q3d2Q", geo, off)
        off += 56
        node_cells.append(rec[5])
    off += nb * 92 + ni * 96
    for _ in range(nbnd):
        (n,) = u64()
        off += 8 * n
    off += 4 * nbnd
    off += 8 * sum(links) + 8 * sum(node_cells)
    return off


def read_result(data: bytes, geo: bytes, cell_nb: int):
    """(names, (t_0, t_max, dt_map), times, frames [n_frames x cell_nb x n_values]); raises on a
    file whose length is not header + whole frames."""
    off = geometry_prefix_length(geo)
    assert data[:off] == geo[:off]
    (nvar,) = struct.unpack_from("<Q", data, off)
    off += 8
    names = []
    for _ in range(nvar):
        (n,) = struct.unpack_from("<Q", data, off)
        off += 8
        names.append(data[off:off + n].decode())
        off += n
    t0, tmax, dtmap = struct.unpack_from("<3d", data, off)
    off += 24
    frame = 8 + 8 * cell_nb * nvar
    rest = len(data) - off
    assert rest % frame == 0, (rest, frame)
    k = rest // frame
    arr = np.frombuffer(data, dtype="<f8", count=k * frame // 8, offset=off).reshape(k, frame // 8)
    return names, (t0, tmax, dtmap), arr[:, 0].copy(), arr[:, 1:].reshape(k, cell_nb, nvar).copy()
