"""Reader and writer of the reference's ``triples.restart`` file.

GAMESS writes the (T) inputs after CCSD as a Fortran unformatted sequential
file that ``program.F90:42-49,195-223`` reads back:

    record 1: no           (8-byte integer under -sdefault64)
    record 2: nu
    record 3: eh(no)       record 4: ep(nu)      record 5: t1(no*nu)
    record 6: t2(nu*nu*no*no)                    record 7: vm(no*no*no*nu)
    record 8: voe(nu*nu*no*no)
    records 9 .. 8+no*nu: one packed VVVO column of nutr = nu(nu+1)/2 doubles each

Every record is framed by a length marker before and after it.  The reference
runs used 4-byte markers (the recorded file sizes only fit that, see
``restart_file_size``); ``read`` detects 4- or 8-byte markers.
"""
from __future__ import annotations

import pathlib
import struct

import numpy as np

from .synthetic import TriplesInputs


def restart_file_size(no: int, nu: int, marker: int = 4, int_bytes: int = 8) -> int:
    """Size in bytes of a triples.restart for (no, nu)."""
    nutr = nu * (nu + 1) // 2
    doubles = no + nu + no * nu + 2 * nu * nu * no * no + no ** 3 * nu + no * nu * nutr
    records = 8 + no * nu
    return doubles * 8 + 2 * int_bytes + records * 2 * marker


def _write_record(fh, payload: bytes, marker: int):
    fmt = "<i" if marker == 4 else "<q"
    n = struct.pack(fmt, len(payload))
    fh.write(n)
    fh.write(payload)
    fh.write(n)


def write(path, inp: TriplesInputs, marker: int = 4) -> int:
    """Write ``inp`` as a triples.restart; returns the file size."""
    path = pathlib.Path(path)
    no, nu = inp.no, inp.nu
    nutr = nu * (nu + 1) // 2
    with open(path, "wb") as fh:
        _write_record(fh, struct.pack("<q", no), marker)
        _write_record(fh, struct.pack("<q", nu), marker)
        for a in (inp.eh, inp.ep, inp.t1, inp.t2, inp.vm, inp.voe):
            _write_record(fh, np.ascontiguousarray(a, dtype="<f8").tobytes(), marker)
        cols = inp.vvvo.reshape(no * nu, nutr)
        for j in range(no * nu):
            _write_record(fh, np.ascontiguousarray(cols[j], dtype="<f8").tobytes(), marker)
    return path.stat().st_size


class RestartFormatError(ValueError):
    pass


def _detect_marker(buf: bytes) -> int:
    # first record holds one 8-byte integer, so it is framed by markers reading 8
    # at offsets (0, 12) with 4-byte markers or (0, 16) with 8-byte markers
    if len(buf) >= 16 and struct.unpack_from("<i", buf, 0)[0] == 8 and struct.unpack_from("<i", buf, 12)[0] == 8:
        return 4
    if len(buf) >= 24 and struct.unpack_from("<q", buf, 0)[0] == 8 and struct.unpack_from("<q", buf, 16)[0] == 8:
        return 8
    raise RestartFormatError("not a triples.restart: first record is not one 8-byte integer")


def read(path) -> TriplesInputs:
    """Read a triples.restart (4- or 8-byte record markers) into TriplesInputs.
    Raises RestartFormatError on a malformed file, as the reference stops with
    "error reading restart file" (program.F90:221-223)."""
    buf = pathlib.Path(path).read_bytes()
    marker = _detect_marker(buf)
    fmt = "<i" if marker == 4 else "<q"
    pos = 0

    def record(expect_bytes: int) -> memoryview:
        nonlocal pos
        if pos + marker > len(buf):
            raise RestartFormatError("error reading restart file: truncated")
        (n,) = struct.unpack_from(fmt, buf, pos)
        if n != expect_bytes:
            raise RestartFormatError(f"error reading restart file: record of {n} bytes, expected {expect_bytes}")
        start = pos + marker
        end = start + n
        if end + marker > len(buf) or struct.unpack_from(fmt, buf, end)[0] != n:
            raise RestartFormatError("error reading restart file: bad record trailer")
        pos = end + marker
        return memoryview(buf)[start:end]

    no = struct.unpack("<q", record(8))[0]
    nu = struct.unpack("<q", record(8))[0]
    if no < 1 or nu < 1:
        raise RestartFormatError(f"error reading restart file: no={no}, nu={nu}")
    nutr = nu * (nu + 1) // 2
    arr = lambda n: np.frombuffer(record(8 * n), dtype="<f8").astype(np.float64)
    eh, ep, t1 = arr(no), arr(nu), arr(no * nu)
    t2, vm, voe = arr(nu * nu * no * no), arr(no ** 3 * nu), arr(nu * nu * no * no)
    vvvo = np.empty((no * nu, nutr))
    for j in range(no * nu):
        vvvo[j] = arr(nutr)
    if pos != len(buf):
        raise RestartFormatError("error reading restart file: trailing bytes")
    return TriplesInputs(no=no, nu=nu, eh=eh, ep=ep, t1=t1, t2=t2, vm=vm, voe=voe, vvvo=vvvo.ravel(),
                         name=pathlib.Path(path).name)
