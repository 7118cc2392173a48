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
``restart_file_size``); ``read`` detects 4- or 8-byte markers.  With 4-byte
markers gfortran splits a record longer than 2,147,483,639 bytes into
subrecords: a negative leading marker means another subrecord follows, a
negative trailing marker that one came before (large T2/VOE records, e.g.
no=40, nu=500, take this form).
"""
from __future__ import annotations

import pathlib
import struct

import numpy as np

from .synthetic import TriplesInputs


# longest subrecord gfortran writes with 4-byte markers
MAX_SUBRECORD = 2_147_483_639


def _subrecords(nbytes: int, marker: int, max_sub: int) -> int:
    return 1 if marker == 8 or nbytes <= max_sub else -(-nbytes // max_sub)


def restart_file_size(no: int, nu: int, marker: int = 4, int_bytes: int = 8, max_sub: int = MAX_SUBRECORD) -> int:
    """Size in bytes of a triples.restart for (no, nu)."""
    nutr = nu * (nu + 1) // 2
    payloads = [int_bytes, int_bytes] + [8 * n for n in (no, nu, no * nu, nu * nu * no * no, no ** 3 * nu,
                                                         nu * nu * no * no)]
    payloads += [8 * nutr] * (no * nu)
    return sum(p + 2 * marker * _subrecords(p, marker, max_sub) for p in payloads)


def _write_record(fh, payload: bytes, marker: int, max_sub: int = MAX_SUBRECORD):
    """One record; with 4-byte markers split into gfortran subrecords of at most
    max_sub bytes (leading marker negative while more follow, trailing marker
    negative on every subrecord after the first)."""
    fmt = "<i" if marker == 4 else "<q"
    if marker == 8 or len(payload) <= max_sub:
        n = struct.pack(fmt, len(payload))
        fh.write(n)
        fh.write(payload)
        fh.write(n)
        return
    view = memoryview(payload)
    nsub = _subrecords(len(payload), marker, max_sub)
    for q in range(nsub):
        part = view[q * max_sub:(q + 1) * max_sub]
        fh.write(struct.pack(fmt, -len(part) if q < nsub - 1 else len(part)))
        fh.write(part)
        fh.write(struct.pack(fmt, -len(part) if q > 0 else len(part)))


def write(path, inp: TriplesInputs, marker: int = 4, max_sub: int = MAX_SUBRECORD) -> int:
    """Write ``inp`` as a triples.restart; returns the file size.  ``max_sub``
    is the subrecord limit of 4-byte markers (gfortran's by default)."""
    path = pathlib.Path(path)
    no, nu = inp.no, inp.nu
    nutr = nu * (nu + 1) // 2
    with open(path, "wb") as fh:
        _write_record(fh, struct.pack("<q", no), marker, max_sub)
        _write_record(fh, struct.pack("<q", nu), marker, max_sub)
        for a in (inp.eh, inp.ep, inp.t1, inp.t2, inp.vm, inp.voe):
            _write_record(fh, np.ascontiguousarray(a, dtype="<f8").tobytes(), marker, max_sub)
        cols = inp.vvvo.reshape(no * nu, nutr)
        for j in range(no * nu):
            _write_record(fh, np.ascontiguousarray(cols[j], dtype="<f8").tobytes(), marker, max_sub)
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

    def record(expect_bytes: int):
        nonlocal pos
        parts, total, first = [], 0, True
        while True:
            if pos + marker > len(buf):
                raise RestartFormatError("error reading restart file: truncated")
            (head,) = struct.unpack_from(fmt, buf, pos)
            n = abs(head)
            start = pos + marker
            end = start + n
            if end + marker > len(buf):
                raise RestartFormatError("error reading restart file: truncated")
            (tail,) = struct.unpack_from(fmt, buf, end)
            # trailing marker: +n on the first subrecord, -n on the ones after it
            if abs(tail) != n or (tail < 0) == first:
                raise RestartFormatError("error reading restart file: bad record trailer")
            parts.append(memoryview(buf)[start:end])
            total += n
            pos = end + marker
            first = False
            if head >= 0:
                break
            if total > expect_bytes:
                break
        if total != expect_bytes:
            raise RestartFormatError(f"error reading restart file: record of {total} bytes, expected {expect_bytes}")
        return parts[0] if len(parts) == 1 else b"".join(parts)

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
