"""NERSC configuration I/O restated with numpy (TEST INFRASTRUCTURE ONLY).

Only tests/ and bench.py's CPU legs use this module, as the checker of the
library's NERSC export/import.  It follows export_config_nersc and
import_config_nersc (field-matrix.h:452-713) and restates the Qlattice and CPS
helpers they call, which are not in the reference tree (Qlattice, jtu fork,
version unpinned): ``fieldCastTruncated`` (first two rows of each link),
``sophisticated_make_to_order`` (global site order x0 fastest),
``from_big_endian_64`` (byte order of every 8-byte word),
``fieldChecksumSum32`` (sum modulo 2^32 of the 32-bit words) and
``field_hash_crc32`` (CRC-32 of the payload; zlib's polynomial, its text
format unpinned, not read by the importer).  Parity unpinned: the reference
ships no NERSC file and cannot run here.  Known answers pin the checksum (the
unit configuration) and zlib pins the CRC.

Deliberate difference: for two-row files the reference computes CHECKSUM after
converting the payload to big-endian (field-matrix.h:476-482), which on a
little-endian host is not the value its own importer checks (on the words after
conversion to host order, field-matrix.h:669-676); it only agrees on a
big-endian host (the BG/Q build of its makefile).  Both formats here use the
importer's definition, so every file written passes import_config_nersc.
"""
from __future__ import annotations

import time
import zlib

import numpy as np

from . import avg_plaquette, reunitarize, volume


class NerscError(Exception):
    """kind: 'io', 'format', 'checksum' or 'plaquette' (where the reference asserts)."""

    def __init__(self, kind: str, msg: str):
        super().__init__(f"{kind}: {msg}")
        self.kind = kind


def avg_real_trace(U: np.ndarray) -> float:
    """avg_real_trace (field-matrix.h:391-405): sum of ReTr over links / (12 V)."""
    return float(np.trace(U, axis1=2, axis2=3).real.sum() / (12.0 * U.shape[0]))


def payload_host(U: np.ndarray, two_row: bool) -> np.ndarray:
    """fieldCastTruncated + make_to_order: links in site order, host byte order."""
    M = U[:, :, :2, :] if two_row else U
    return np.ascontiguousarray(M).view(np.float64).ravel()


def checksum32(host_words: np.ndarray) -> int:
    """fieldChecksumSum32: sum modulo 2^32 of the 32-bit words (host byte order)."""
    return int(np.ascontiguousarray(host_words).view(np.uint32).astype(np.uint64).sum() & 0xFFFFFFFF)


def crc32(host_words: np.ndarray) -> int:
    return zlib.crc32(np.ascontiguousarray(host_words).tobytes()) & 0xFFFFFFFF


def format_header(dims, two_row, crc, csum, link_trace, plaq, label, seq, beta, unix_time) -> str:
    """The header lines of field-matrix.h:486-508 / :530-552, in that order."""
    g = (lambda x: "%.12g" % x) if two_row else (lambda x: "%g" % x)
    lines = ["BEGIN_HEADER", "HDR_VERSION = 1.0",
             "DATATYPE = 4D_SU3_GAUGE" if two_row else "DATATYPE = 4D_SU3_GAUGE_3x3"]
    lines += [f"DIMENSION_{d + 1} = {int(dims[d])}" for d in range(4)]
    lines += [f"CRC32HASH = {crc:x}", f"CHECKSUM = {csum:x}", "LINK_TRACE = " + g(link_trace),
              "PLAQUETTE = " + g(plaq), "CREATOR = RBC", "ARCHIVE_DATE = " + time.ctime(unix_time),
              "ENSEMBLE_LABEL = " + label, "FLOATING_POINT = IEEE64BIG", "ENSEMBLE_ID = NOT yet implemented",
              f"SEQUENCE_NUMBER = {int(seq)}", "BETA = " + g(beta), "END_HEADER"]
    return "\n".join(lines) + "\n"


def export_config(path, dims, U, two_row=True, beta=2.25, seq=0, label="", unix_time=None) -> dict:
    """export_config_nersc (field-matrix.h:452-572)."""
    host = payload_host(U, two_row)
    csum, crc = checksum32(host), crc32(host)
    plaq, tr = avg_plaquette(dims, U), avg_real_trace(U)
    t = int(time.time()) if unix_time is None else int(unix_time)
    hdr = format_header(dims, two_row, crc, csum, tr, plaq, label, seq, beta, t)
    with open(path, "wb") as f:
        f.write(hdr.encode())
        f.write(host.astype(">f8").tobytes())
    return {"checksum": csum, "crc32": crc, "plaquette": plaq, "link_trace": tr, "payload_offset": len(hdr)}


def _snatch(line: str, key: str):
    """snatch_keyword (field-matrix.h:575-592)."""
    if key not in line:
        return None
    i = line.find("=")
    if i < 0:
        raise NerscError("format", f"{key} line without '='")
    v = line[i + 1:].lstrip(" \t")
    return v[:-1] if v.endswith("\n") else v


def read_header(path) -> dict:
    h = {"datatype": None, "dims": [0, 0, 0, 0], "checksum": 0, "plaquette": 0.0, "payload_offset": -1}
    try:
        f = open(path, "rb")
    except OSError as e:
        raise NerscError("io", str(e))
    with f:
        while True:
            raw = f.readline()
            if not raw:
                break
            line = raw.decode("latin-1")
            v = _snatch(line, "DATATYPE")
            if v is not None:
                h["datatype"] = v
            for d in range(4):
                v = _snatch(line, f"DIMENSION_{d + 1}")
                if v is not None:
                    h["dims"][d] = int(v.split()[0]) if v.split() else 0
            v = _snatch(line, "CHECKSUM")
            if v is not None:
                try:
                    h["checksum"] = int(v.split()[0], 16) & 0xFFFFFFFF
                except (ValueError, IndexError):
                    raise NerscError("format", "unreadable CHECKSUM")
            v = _snatch(line, "PLAQUETTE")
            if v is not None:
                h["plaquette"] = float(v.split()[0]) if v.split() else 0.0
            if "END_HEADER" in line:
                h["payload_offset"] = f.tell()
                break
    if h["payload_offset"] < 0:
        raise NerscError("format", "no END_HEADER line")
    if h["datatype"] == "4D_SU3_GAUGE":
        h["two_row"] = True
    elif h["datatype"] == "4D_SU3_GAUGE_3x3":
        h["two_row"] = False
    else:
        raise NerscError("format", f"WRONG DATATYPE {h['datatype']!r}")
    return h


def import_config(path, dims):
    """import_config_nersc (field-matrix.h:594-713): returns (U, info)."""
    h = read_header(path)
    if list(h["dims"]) != [int(d) for d in dims]:
        raise NerscError("format", "WRONG Lattice Size")
    V = volume(dims)
    nc = 6 if h["two_row"] else 9
    with open(path, "rb") as f:
        f.seek(h["payload_offset"])
        raw = f.read(V * 4 * nc * 16)
    if len(raw) != V * 4 * nc * 16:
        raise NerscError("format", "payload shorter than the lattice needs")
    host = np.frombuffer(raw, ">f8").astype(np.float64)
    csum = checksum32(host)
    info = {"checksum": csum, "crc32": crc32(host), "checksum_header": h["checksum"],
            "plaquette_header": h["plaquette"], "two_row": h["two_row"]}
    if csum != h["checksum"]:
        raise NerscError("checksum", f"{h['checksum']:x}(labeled) vs {csum:x}(computed)")
    M = host.view(np.complex128).reshape(V, 4, nc // 3, 3)
    U = np.zeros((V, 4, 3, 3), np.complex128)
    U[:, :, : nc // 3, :] = M
    if h["two_row"]:
        U, _ = reunitarize(dims, U)
    plaq = avg_plaquette(dims, U)
    info["plaquette"] = plaq
    info["link_trace"] = avg_real_trace(U)
    if abs(plaq - h["plaquette"]) > 1e-4:
        raise NerscError("plaquette", f"{h['plaquette']:.8f}(labeled) vs {plaq:.8f}(computed)")
    return U, info
