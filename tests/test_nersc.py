"""NERSC configuration I/O (export_config_nersc / import_config_nersc,
field-matrix.h:452-713): the numpy oracle, the host header reader of the
library, and (gpu) the device load/save path against the oracle.

Bars: payload bytes, CHECKSUM and CRC32HASH bit-exact; links of 3x3 files
bit-exact; links of two-row files (third row rebuilt by reunitarize) within
1e-15; plaquette and link trace within 1e-12.
"""
import os
import zlib

import numpy as np
import pytest

import mag_b200 as M
import oracle as O
from mag_b200 import _lib
from mag_b200.field_hmc import crc32_segmented, read_nersc_header
from oracle import nersc as N

DIMS = (4, 4, 4, 6)


def _payload_bytes(path, offset):
    with open(path, "rb") as f:
        f.seek(offset)
        return f.read()


# ------------------------------------------------------------------ CPU
@pytest.mark.parametrize("two_row", [True, False])
def test_oracle_roundtrip(tmp_path, two_row):
    U = O.gen_hot(DIMS, 3)
    p = tmp_path / "cfg.nersc"
    w = N.export_config(p, DIMS, U, two_row=two_row, beta=2.25, seq=7, label="t")
    U2, info = N.import_config(p, DIMS)
    assert info["checksum"] == w["checksum"] and info["crc32"] == w["crc32"]
    if two_row:
        assert np.abs(U2 - U).max() < 1e-14
    else:
        assert np.array_equal(U2, U)
    hdr = open(p, "rb").read(w["payload_offset"]).decode()
    keys = [ln.split(" = ")[0] for ln in hdr.splitlines()]
    assert keys == ["BEGIN_HEADER", "HDR_VERSION", "DATATYPE", "DIMENSION_1", "DIMENSION_2", "DIMENSION_3",
                    "DIMENSION_4", "CRC32HASH", "CHECKSUM", "LINK_TRACE", "PLAQUETTE", "CREATOR", "ARCHIVE_DATE",
                    "ENSEMBLE_LABEL", "FLOATING_POINT", "ENSEMBLE_ID", "SEQUENCE_NUMBER", "BETA", "END_HEADER"]
    payload = _payload_bytes(p, w["payload_offset"])
    assert len(payload) == O.volume(DIMS) * 4 * (6 if two_row else 9) * 16
    assert zlib.crc32(np.frombuffer(payload, ">f8").astype(np.float64).tobytes()) == w["crc32"]


@pytest.mark.parametrize("two_row", [True, False])
def test_unit_configuration_known_answer(tmp_path, two_row):
    """Unit links: every 1.0 is the word pair (0x00000000, 0x3FF00000) in host
    order, zeros add nothing, so CHECKSUM = 4 V (2 or 3) 0x3FF00000 mod 2^32."""
    U = O.gen_cold(DIMS)
    w = N.export_config(tmp_path / "unit", DIMS, U, two_row=two_row)
    V = O.volume(DIMS)
    assert w["checksum"] == (4 * V * (2 if two_row else 3) * 0x3FF00000) % (1 << 32)
    assert w["plaquette"] == 1.0 and w["link_trace"] == 1.0


def test_crc_segment_chaining_host():
    rng = np.random.default_rng(0)
    for n in (0, 1, 17, 4096, 16384, 16400, 99999):
        d = rng.integers(0, 256, n, dtype=np.uint8).tobytes()
        for seg in (16, 48, 16384):
            assert crc32_segmented(d, seg) == zlib.crc32(d)


@pytest.mark.parametrize("two_row", [True, False])
def test_library_header_reader(tmp_path, two_row):
    U = O.gen_hot(DIMS, 4)
    p = tmp_path / "cfg"
    w = N.export_config(p, DIMS, U, two_row=two_row)
    h = read_nersc_header(p)
    assert h["dims"] == list(DIMS) and h["two_row"] == int(two_row)
    assert h["checksum_header"] == w["checksum"] and h["crc32_header"] == w["crc32"]
    assert h["payload_offset"] == w["payload_offset"]
    # PLAQUETTE is written with 12 significant digits (two-row) or 6 (3x3)
    assert h["plaquette_header"] == float(("%.12g" if two_row else "%g") % w["plaquette"])


def _write(p, text, payload=b""):
    with open(p, "wb") as f:
        f.write(text.encode())
        f.write(payload)


def test_library_header_errors(tmp_path):
    with pytest.raises(M.MagError) as e:
        read_nersc_header(tmp_path / "missing")
    assert e.value.code == _lib.MAG_ERR_IO
    _write(tmp_path / "noend", "BEGIN_HEADER\nDATATYPE = 4D_SU3_GAUGE\n")
    with pytest.raises(M.MagError) as e:
        read_nersc_header(tmp_path / "noend")
    assert e.value.code == _lib.MAG_ERR_FORMAT
    _write(tmp_path / "type", "BEGIN_HEADER\nDATATYPE = 4D_SU3_GAUGE_2x3\nEND_HEADER\n")
    with pytest.raises(M.MagError) as e:
        read_nersc_header(tmp_path / "type")
    assert e.value.code == _lib.MAG_ERR_FORMAT and "DATATYPE" in str(e.value)
    _write(tmp_path / "csum", "BEGIN_HEADER\nDATATYPE = 4D_SU3_GAUGE\nCHECKSUM = zz\nEND_HEADER\n")
    with pytest.raises(M.MagError) as e:
        read_nersc_header(tmp_path / "csum")
    assert e.value.code == _lib.MAG_ERR_FORMAT
    # the reference only strips '\n': a CRLF header carries '\r' into DATATYPE and is rejected
    _write(tmp_path / "crlf", "BEGIN_HEADER\r\nDATATYPE = 4D_SU3_GAUGE\r\nEND_HEADER\r\n")
    with pytest.raises(M.MagError) as e:
        read_nersc_header(tmp_path / "crlf")
    assert e.value.code == _lib.MAG_ERR_FORMAT
    with pytest.raises(N.NerscError):
        N.read_header(tmp_path / "crlf")


def test_oracle_detects_corruption(tmp_path):
    U = O.gen_hot(DIMS, 6)
    p = tmp_path / "cfg"
    w = N.export_config(p, DIMS, U, two_row=False)
    raw = bytearray(open(p, "rb").read())
    raw[w["payload_offset"] + 100] ^= 0x10
    open(tmp_path / "bad", "wb").write(raw)
    with pytest.raises(N.NerscError) as e:
        N.import_config(tmp_path / "bad", DIMS)
    assert e.value.kind == "checksum"


# ------------------------------------------------------------------ GPU
@pytest.mark.gpu
@pytest.mark.parametrize("two_row", [True, False])
def test_load_matches_oracle(tmp_path, two_row):
    U = O.gen_hot(DIMS, 11)
    p = tmp_path / "cfg"
    w = N.export_config(p, DIMS, U, two_row=two_row, beta=2.25, seq=3, label="x")
    Uo, io = N.import_config(p, DIMS)
    with M.Chmc(DIMS) as c:
        info = c.import_config_nersc(p)
        Ug = c.get_gauge()
    assert info["checksum"] == info["checksum_header"] == w["checksum"]
    assert info["crc32"] == w["crc32"]
    if two_row:
        assert np.abs(Ug - Uo).max() < 1e-15
    else:
        assert np.array_equal(Ug, Uo)
    assert abs(info["plaquette"] - io["plaquette"]) < 1e-12
    assert abs(info["link_trace"] - io["link_trace"]) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("two_row", [True, False])
def test_save_matches_oracle(tmp_path, two_row):
    with M.Chmc(DIMS, seed=5) as c:
        c.hot_start(9)
        U = c.get_gauge()
        info = c.export_config_nersc(tmp_path / "gpu", beta=2.37, sequence_num=12, ensemble_label="ens",
                                     skip_third=two_row)
    w = N.export_config(tmp_path / "cpu", DIMS, U, two_row=two_row, beta=2.37, seq=12, label="ens")
    assert _payload_bytes(tmp_path / "gpu", info["payload_offset"]) == _payload_bytes(tmp_path / "cpu",
                                                                                       w["payload_offset"])
    assert info["checksum"] == w["checksum"] and info["crc32"] == w["crc32"]
    assert abs(info["plaquette"] - w["plaquette"]) < 1e-12 and abs(info["link_trace"] - w["link_trace"]) < 1e-12
    hg = N.read_header(tmp_path / "gpu")
    assert hg["checksum"] == w["checksum"] and hg["dims"] == list(DIMS) and hg["two_row"] == two_row
    # the oracle importer accepts the library's file, and vice versa
    N.import_config(tmp_path / "gpu", DIMS)
    with M.Chmc(DIMS) as c2:
        c2.import_config_nersc(tmp_path / "cpu")


@pytest.mark.gpu
def test_load_errors(tmp_path):
    U = O.gen_hot(DIMS, 12)
    p = tmp_path / "cfg"
    w = N.export_config(p, DIMS, U, two_row=False)
    raw = open(p, "rb").read()
    with M.Chmc(DIMS) as c:
        c.cold_start()
        before = c.get_gauge()
        # flipped payload bit: checksum error, links untouched
        bad = bytearray(raw)
        bad[w["payload_offset"] + 8 * 37 + 3] ^= 0x01
        open(tmp_path / "bit", "wb").write(bad)
        with pytest.raises(M.MagError) as e:
            c.import_config_nersc(tmp_path / "bit")
        assert e.value.code == _lib.MAG_ERR_CHECKSUM
        assert np.array_equal(c.get_gauge(), before)
        # short payload
        open(tmp_path / "short", "wb").write(raw[:-16])
        with pytest.raises(M.MagError) as e:
            c.import_config_nersc(tmp_path / "short")
        assert e.value.code == _lib.MAG_ERR_FORMAT
        # wrong plaquette in the header: the links load, the call reports the mismatch
        hdr = raw[:w["payload_offset"]].decode()
        line = next(ln for ln in hdr.splitlines() if ln.startswith("PLAQUETTE"))
        hdr2 = hdr.replace(line, "PLAQUETTE = 0.5")
        open(tmp_path / "plaq", "wb").write(hdr2.encode() + raw[w["payload_offset"]:])
        with pytest.raises(M.MagError) as e:
            c.import_config_nersc(tmp_path / "plaq")
        assert e.value.code == _lib.MAG_ERR_PLAQUETTE
        assert np.array_equal(c.get_gauge(), U)
    with M.Chmc((4, 4, 4, 4)) as c:
        with pytest.raises(M.MagError) as e:
            c.import_config_nersc(p)
        assert e.value.code == _lib.MAG_ERR_FORMAT and "Lattice Size" in str(e.value)


@pytest.mark.gpu
@pytest.mark.parametrize("two_row,dims", [(True, (16, 16, 16, 32)), (False, (16, 16, 16, 32)),
                                          (False, (24, 24, 24, 24))])
def test_roundtrip_full_size(tmp_path, two_row, dims):
    """16^3 x 32 and 24^4 (payload 50-191 MB: many 8 MB pipeline chunks, the
    24^4 file more chunks than pinned slots, so every slot is reused):
    save -> load is exact (3x3) or a fixed point of reunitarize (two-row), and
    the file's digests equal zlib / numpy over the payload."""
    p = tmp_path / "big"
    with M.Chmc(dims, seed=2) as c:
        c.hot_start(4)
        U = c.get_gauge()
        si = c.export_config_nersc(p, skip_third=two_row)
        li = c.import_config_nersc(p)
        U2 = c.get_gauge()
    assert li["checksum"] == si["checksum"] and li["crc32"] == si["crc32"]
    host = np.frombuffer(_payload_bytes(p, si["payload_offset"]), ">f8").astype(np.float64)
    assert N.checksum32(host) == si["checksum"] and N.crc32(host) == si["crc32"]
    if two_row:
        assert np.abs(U2 - U).max() < 1e-14
    else:
        assert np.array_equal(U2, U)


@pytest.mark.gpu
def test_ensemble_chain_io(tmp_path):
    chains = [dict(dims=(4, 4, 4, 4), beta=2.1), dict(dims=(4, 4, 4, 6), beta=2.3)]
    with M.Chmc(chains=chains, seed=3) as c:
        c.hot_start(8)
        U1 = c.get_gauge(1)
        c.export_config_nersc(tmp_path / "c1", chain=1, skip_third=False)
    with M.Chmc(chains=[dict(dims=(4, 4, 4, 6))]) as d:
        d.import_config_nersc(tmp_path / "c1")
        assert np.array_equal(d.get_gauge(), U1)
