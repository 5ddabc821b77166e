"""Gauge-configuration files (b200dwf.gauge_io) against the reference's own
readers and writers (tests/golden/gauge_io.npz: SHA-256 digests of what the
reference corelib produced from the same synthetic text configuration):
Text_4x4x4x8 tiled onto a larger lattice, Binary (ILDG order, big-endian)
written byte for byte, and read back."""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))


def _golden():
    z = np.load(os.path.join(HERE, "golden", "gauge_io.npz"))
    return json.loads(str(z["meta"])), json.loads(str(z["digest"]))


def test_text_and_binary_match_the_reference(tmp_path):
    from b200dwf import gauge_io
    from make_golden import io_text
    meta, digest = _golden()
    text = tmp_path / "conf.txt"
    text.write_text(io_text(meta))
    u = gauge_io.read_text_4x4x4x8(str(text), meta["lattice"])
    assert hashlib.sha256(u.astype("<f8").tobytes()).hexdigest() == digest["text_read.bin"]
    out = tmp_path / "conf.bin"
    gauge_io.write_binary(str(out), u, meta["lattice"])
    assert hashlib.sha256(out.read_bytes()).hexdigest() == digest["conf.bin"]
    back = gauge_io.read_binary(str(out), meta["lattice"])
    assert hashlib.sha256(back.astype("<f8").tobytes()).hexdigest() == digest["bin_read.bin"]
    assert np.array_equal(back, u)


def test_tiling_and_size_checks(tmp_path):
    """Every 4x4x4x8 block of the tiled configuration is the file's; short
    files and wrong sizes are rejected."""
    import pytest
    from b200dwf import gauge_io
    from make_golden import io_text
    meta, _ = _golden()
    text = tmp_path / "conf.txt"
    text.write_text(io_text(meta))
    small = gauge_io.read_text_4x4x4x8(str(text), [4, 4, 4, 8])
    big = gauge_io.read_text_4x4x4x8(str(text), [8, 8, 4, 16])
    s = small.reshape(4, 8, 4, 4, 4, 18)          # [mu][t][z][y][x][r]
    b = big.reshape(4, 16, 4, 8, 8, 18)
    for dt in (0, 8):
        for dy in (0, 4):
            for dx in (0, 4):
                assert np.array_equal(b[:, dt:dt + 8, :, dy:dy + 4, dx:dx + 4], s)
    short = tmp_path / "short.txt"
    short.write_text("\n".join(text.read_text().split("\n")[:100]))
    with pytest.raises(ValueError):
        gauge_io.read_text_4x4x4x8(str(short), [4, 4, 4, 8])
    with pytest.raises(ValueError):
        gauge_io.write_binary(str(tmp_path / "x.bin"), small, [8, 4, 4, 8])
    gauge_io.write_binary(str(tmp_path / "y.bin"), small, [4, 4, 4, 8])
    with pytest.raises(ValueError):
        gauge_io.read_binary(str(tmp_path / "y.bin"), [8, 4, 4, 8])
