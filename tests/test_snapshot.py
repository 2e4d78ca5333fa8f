"""snapshot_v3 I/O on the host (no GPU): the byte layout of the reference's
format (src/snapshot_v3.rs:12-47 header fields in order, little-endian,
408 bytes; 36-byte particles, sign 1 / 255), written by the library and read
back, and a file built here field by field read by the library."""
import struct

import numpy as np

import janus_treepm as J

HDR = "<QIIQ" + "d" * 10 + "II" + "d" + "Q" + "ddd" + "256s"


def _particles(n, seed=3):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-10, 10, (n, 3)).astype(np.float32)
    vel = rng.normal(0, 1, (n, 3)).astype(np.float32)
    sg = np.where(rng.random(n) < 0.4, 1, -1).astype(np.int8)
    mass = np.where(sg > 0, 1.5, 28.5).astype(np.float32)
    eps = np.full(n, 0.05, np.float32)
    return pos, vel, sg, mass, eps


def test_write_layout_is_the_reference_format(tmp_path):
    pos, vel, sg, mass, eps = _particles(1000)
    meta = J.snapshot_meta(a=0.2, t_gyr=1.5, h0=70.0, omega_b=0.04, z_init=99.0, z_start_run=4.0,
                           seed_ic=7, run_label="janus-b200 test")
    path = tmp_path / "snap.bin"
    J.snapshot_write(path, meta, 20.0, 19.0, pos, vel, sg, mass, eps)
    raw = path.read_bytes()
    assert struct.calcsize(HDR) == 408 and len(raw) == 408 + 36 * 1000
    h = struct.unpack(HDR, raw[:408])
    assert h[0] == 0x0A335653554E414A and h[1] == 3 and h[2] == 408 and h[3] == 1000
    assert raw[:8] == b"JANUSV3\n"
    a, t, L, h0, mu, ob, mp, mm, ep, em = h[4:14]
    assert (a, t, L, h0, mu, ob) == (0.2, 1.5, 20.0, 70.0, 19.0, 0.04)
    assert np.float32(mp) == np.float32(1.5) and np.float32(mm) == np.float32(28.5)
    assert h[15] == 7 and h[16] == 99.0 and h[18] == 4.0
    assert h[21].rstrip(b"\0") == b"janus-b200 test"
    rec = np.frombuffer(raw[408:], dtype=np.dtype([("pos", "<f4", 3), ("vel", "<f4", 3), ("mass", "<f4"),
                                                   ("eps", "<f4"), ("sign", "u1"), ("lvl", "u1"),
                                                   ("star", "u1"), ("flags", "u1")]))
    assert np.array_equal(rec["pos"], pos) and np.array_equal(rec["vel"], vel)
    assert np.array_equal(rec["sign"], np.where(sg > 0, 1, 255))
    assert np.array_equal(rec["mass"], mass) and not rec["lvl"].any()


def test_read_a_file_built_field_by_field(tmp_path):
    pos, vel, sg, mass, eps = _particles(257, seed=5)
    label = b"built by hand"
    hdr = struct.pack(HDR, 0x0A335653554E414A, 3, 408, 257, 0.5, 2.0, 50.0, 67.0, 5.0, 0.05,
                      1.0, 5.0, 0.1, 0.2, 0, 11, 30.0, 0, 30.0, 0.0, 0.0, label)
    body = b"".join(struct.pack("<8f4B", *pos[i], *vel[i], mass[i], eps[i], 1 if sg[i] > 0 else 255, 0, 0, 0)
                    for i in range(257))
    path = tmp_path / "hand.bin"
    path.write_bytes(hdr + body)
    meta, L, mu, p2, v2, s2, m2, e2 = J.snapshot_read(path)
    assert (L, mu, meta.a, meta.t_gyr, meta.seed_ic, meta.z_init) == (50.0, 5.0, 0.5, 2.0, 11, 30.0)
    assert meta.run_label == label
    assert np.array_equal(p2, pos) and np.array_equal(v2, vel) and np.array_equal(s2, sg)
    assert np.array_equal(m2, mass) and np.array_equal(e2, eps)


def test_bad_magic_is_rejected(tmp_path):
    path = tmp_path / "bad.bin"
    path.write_bytes(b"NOTASNAP" + bytes(500))
    L = J.library()
    import ctypes as C
    n = C.c_size_t()
    assert L.jt_snapshot_read(str(path).encode(), None, None, None, None, None, None, None, None, 0,
                              C.byref(n)) == J.JT_EINVAL


def test_raw_driver_format(tmp_path):
    """save_snapshot of the production driver
    (src/bin/janus_mu19_production.rs:198-216): 16-byte header, 25-byte
    records."""
    pos, vel, sg, _, _ = _particles(333, seed=9)
    path = tmp_path / "raw.bin"
    J.snapshot_write_raw(path, pos, vel, sg, 250.0, 1234, 3.5)
    raw = path.read_bytes()
    assert len(raw) == 16 + 25 * 333
    assert struct.unpack("<IfIf", raw[:16]) == (333, 250.0, 1234, 3.5)
    rec = np.frombuffer(raw[16:], dtype=np.dtype([("pos", "<f4", 3), ("vel", "<f4", 3), ("sign", "i1")]))
    assert np.array_equal(rec["pos"], pos) and np.array_equal(rec["vel"], vel)
    assert np.array_equal(rec["sign"], sg)
    p2, v2, s2, box, step, z = J.snapshot_read_raw(path)
    assert (box, step, z) == (250.0, 1234, 3.5)
    assert np.array_equal(p2, pos) and np.array_equal(v2, vel) and np.array_equal(s2, sg)
