"""PMSH mesh files (the reference's binary mesh format) read on the host: files written by the
reference's own MeshIO::writeBinary decode to the reference's arrays; malformed files are rejected."""
import os
import struct

import numpy as np
import pytest

from conftest import GOLDEN, golden, load_package


@pytest.mark.parametrize("name,nsd,order,family", [("block_q2_hex_3x2x2", 3, 2, 2), ("block_q1_quad_5x4", 2, 1, 0)])
def test_reads_the_reference_writer(name, nsd, order, family):
    rsd = load_package()
    info, xyz, ien, rng = rsd.read_pmsh(os.path.join(GOLDEN, name + ".pmsh"))
    g = golden(name + ".npz")
    assert info["spatial_dim"] == info["parametric_dim"] == nsd
    assert info["family"] == family and info["basis"] == 0 and info["iga"] == 0
    assert info["order"] == [order] * nsd
    assert np.array_equal(xyz, g["xyz"]) and np.array_equal(ien, g["ien"]) and np.array_equal(rng, g["rng"])


def test_rejects_malformed_files(tmp_path):
    rsd = load_package()
    good = open(os.path.join(GOLDEN, "block_q1_quad_5x4.pmsh"), "rb").read()
    cases = {
        "magic": b"XXXX" + good[4:],
        "version": good[:4] + struct.pack("<I", 7) + good[8:],
        "truncated": good[:-10],
        "node": None,
    }
    # a connectivity entry pointing past the last node
    info, xyz, ien, rng = rsd.read_pmsh(os.path.join(GOLDEN, "block_q1_quad_5x4.pmsh"))
    off = len(good) - 4 * rng.size - 8 * ien.size
    cases["node"] = good[:off] + struct.pack("<Q", 10 ** 6) + good[off + 8:]
    for key, data in cases.items():
        p = tmp_path / f"{key}.pmsh"
        p.write_bytes(data)
        with pytest.raises(rsd.RsdError) as e:
            rsd.read_pmsh(str(p))
        assert e.value.code == -1, key
    with pytest.raises(rsd.RsdError):
        rsd.read_pmsh(str(tmp_path / "missing.pmsh"))
