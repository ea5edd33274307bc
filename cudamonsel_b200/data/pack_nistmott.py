"""Pack NIST SRD-64 elastic tables (the reference's ``NistXSec/E%02d.D64`` files)
into the little-endian binary this library loads on machines without the
reference tree.

Source layout (parsed by ``EPQLibrary/NISTMottScatteringAngle.cu:44-66``): one
header line (Z), then 61 blocks, each a total cross section in Bohr radii
squared followed by 201 quantiles q(r) at r = 0, 0.005, ..., 1.

Output ``E%02d.bin``: 8-byte magic b"NMOTT001", int32 Z, int32 61, int32 201,
int32 0, then 61 float64 cross sections, then 61*201 float64 quantiles (row j =
energy node j).  Values are the decimal strings parsed to the nearest double,
as ``sciToDub`` does.

    python -m cudamonsel_b200.data.pack_nistmott <NistXSec dir> Z [Z ...]
"""
import os
import struct
import sys

import numpy as np

SPWEM_LEN = 61
X1_LEN = 201


def parse_d64(path):
    with open(path) as f:
        lines = f.read().split("\n")
    z = int(float(lines[0]))
    vals = [float(s) for s in lines[1:1 + SPWEM_LEN * (X1_LEN + 1)]]
    arr = np.array(vals, dtype=np.float64).reshape(SPWEM_LEN, X1_LEN + 1)
    return z, arr[:, 0].copy(), arr[:, 1:].copy()


def write_bin(path, z, spwem, x1):
    with open(path, "wb") as f:
        f.write(b"NMOTT001")
        f.write(struct.pack("<4i", z, SPWEM_LEN, X1_LEN, 0))
        f.write(np.ascontiguousarray(spwem, dtype="<f8").tobytes())
        f.write(np.ascontiguousarray(x1, dtype="<f8").tobytes())


def read_bin(path):
    with open(path, "rb") as f:
        raw = f.read()
    assert raw[:8] == b"NMOTT001", path
    z, n1, n2, _ = struct.unpack("<4i", raw[8:24])
    body = np.frombuffer(raw[24:], dtype="<f8")
    return z, body[:n1].copy(), body[n1:n1 + n1 * n2].reshape(n1, n2).copy()


if __name__ == "__main__":
    src = sys.argv[1]
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "NistXSec")
    os.makedirs(out, exist_ok=True)
    for zs in sys.argv[2:]:
        z = int(zs)
        zz, spwem, x1 = parse_d64(os.path.join(src, "E%02d.D64" % z))
        assert zz == z
        write_bin(os.path.join(out, "E%02d.bin" % z), z, spwem, x1)
        print("packed Z=%d" % z)
