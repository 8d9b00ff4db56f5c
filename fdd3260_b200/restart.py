"""The reference's restart file (src/IO/restarting.f90 savedata :778-1068, readdata
:64-770), version 'V04', for the fields of this path.

The file is Fortran sequential unformatted: every WRITE statement is one record, framed
by a 4-byte little-endian length before and after it (the gfortran and ifort default),
its items packed without padding; `real` is 8 bytes (-r8 / -fdefault-real-8), `integer`
4.  The records in order:

  1. vers                                   character(len=3) 'V04'
  2. time, ntime, dt, ntau, nx, ny, nz, dx, dy, dz, nscal, nparc, xn_ccn0, xn_in0
  3. u00, v00, p0, den0, stab0, n20, g0, avden0, pt0, mse0, t0, qt0, qv0, ql0, nl0, w0,
     k0 (nz each), scal0 (nz, nscal)
  4. one record per field x(1:nx, 1:ny, 1:nz): u, v, w, p, es, qt, dens, the
     hydrometeors (q, n[, w] per class; none without microphysics), scal(:,:,:,h) for
     h = 1..nscal, then turbu%ksgs when with_dif (version > 2; buoy before it for
     versions 1 and 2).

Records longer than 2**31 - 1 bytes (fields above about 268 M cells) are split into
subrecords by the Fortran runtimes; this module rejects them instead of writing a
framing it cannot check here.
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field

import numpy as np

VERS = b"V04"
HEADER = [("time", "d"), ("ntime", "i"), ("dt", "d"), ("ntau", "i"), ("nx", "i"), ("ny", "i"), ("nz", "i"),
          ("dx", "d"), ("dy", "d"), ("dz", "d"), ("nscal", "i"), ("nparc", "i"), ("xn_ccn0", "d"), ("xn_in0", "d")]
PROFILES = ["u00", "v00", "p0", "den0", "stab0", "n20", "g0", "avden0", "pt0", "mse0", "t0", "qt0", "qv0", "ql0",
            "nl0", "w0", "k0"]
MAX_RECORD = 2**31 - 1


@dataclass
class Restart:
    """Content of a restart file: header items, profiles (nz each; scal0 is (nscal, nz)),
    and the fields as arrays of shape (nz, ny, nx) (the Fortran x(1:nx,1:ny,1:nz))."""
    header: dict
    profiles: dict
    fields: dict                          # u, v, w, p, es, qt, dens
    scal: list = field(default_factory=list)
    hydro: list = field(default_factory=list)
    buoy: np.ndarray | None = None
    ksgs: np.ndarray | None = None
    vers: bytes = VERS


def _record(f, payload: bytes) -> None:
    n = len(payload)
    if n > MAX_RECORD:
        raise ValueError(f"record of {n} bytes exceeds the 2 GiB single-record limit")
    f.write(struct.pack("<i", n))
    f.write(payload)
    f.write(struct.pack("<i", n))


def _read_record(f) -> bytes:
    head = f.read(4)
    if len(head) < 4:
        raise EOFError("end of restart file")
    (n,) = struct.unpack("<i", head)
    if n < 0:
        raise ValueError("continued (subrecord) records are not supported")
    payload = f.read(n)
    (m,) = struct.unpack("<i", f.read(4))
    if m != n or len(payload) != n:
        raise ValueError("corrupt record framing")
    return payload


def _field_bytes(a: np.ndarray, shape) -> bytes:
    a = np.ascontiguousarray(a, dtype="<f8")
    if a.shape != shape:
        raise ValueError(f"field shape {a.shape}, expected {shape}")
    return a.tobytes()


def write(path: str, r: Restart) -> None:
    h = r.header
    nx, ny, nz, nscal = h["nx"], h["ny"], h["nz"], h["nscal"]
    shape = (nz, ny, nx)
    with open(path, "wb") as f:
        _record(f, r.vers)
        _record(f, struct.pack("<" + "".join(t for _, t in HEADER), *[h[k] for k, _ in HEADER]))
        prof = [np.ascontiguousarray(r.profiles.get(k, np.zeros(nz)), dtype="<f8") for k in PROFILES]
        scal0 = np.ascontiguousarray(r.profiles.get("scal0", np.zeros((nscal, nz))), dtype="<f8")
        if any(p.shape != (nz,) for p in prof) or scal0.shape != (nscal, nz):
            raise ValueError("profiles must have nz values (scal0: nscal x nz)")
        _record(f, b"".join(p.tobytes() for p in prof) + scal0.tobytes())
        for k in ("u", "v", "w", "p", "es", "qt", "dens"):
            _record(f, _field_bytes(r.fields[k], shape))
        for hyd in r.hydro:
            for a in hyd:
                _record(f, _field_bytes(a, shape))
        if len(r.scal) != nscal:
            raise ValueError("one scal field per nscal")
        for a in r.scal:
            _record(f, _field_bytes(a, shape))
        ivers = int(r.vers[1:3]) if r.vers[:1] == b"V" else 0
        if ivers > 0:
            if ivers <= 2:
                _record(f, _field_bytes(r.buoy if r.buoy is not None else np.zeros(shape), shape))
            if r.ksgs is not None:
                _record(f, _field_bytes(r.ksgs, shape))


def read(path: str, with_dif: bool = False, nhydro_records=()) -> Restart:
    """Read a restart file.  nhydro_records: per hydrometeor class the number of field
    records saved (2, or 3 with the rimed mass), empty without microphysics."""
    with open(path, "rb") as f:
        first = _read_record(f)
        if first[:1] == b"V" and len(first) == 3:
            vers, ivers = first, int(first[1:3])
            hdr = _read_record(f)
        else:   # files without a version record start with the header (readdata :98-101)
            vers, ivers, hdr = b"", 0, first
        vals = struct.unpack("<" + "".join(t for _, t in HEADER), hdr)
        header = dict(zip([k for k, _ in HEADER], vals))
        nx, ny, nz, nscal = header["nx"], header["ny"], header["nz"], header["nscal"]
        shape = (nz, ny, nx)
        pr = np.frombuffer(_read_record(f), dtype="<f8")
        if pr.size != nz * (len(PROFILES) + nscal):
            raise ValueError("profile record does not match nz and nscal")
        profiles = {k: pr[q * nz:(q + 1) * nz].copy() for q, k in enumerate(PROFILES)}
        profiles["scal0"] = pr[len(PROFILES) * nz:].reshape(nscal, nz).copy()

        def fld():
            a = np.frombuffer(_read_record(f), dtype="<f8")
            if a.size != nx * ny * nz:
                raise ValueError("field record does not match nx, ny, nz")
            return a.reshape(shape).copy()

        fields = {k: fld() for k in ("u", "v", "w", "p", "es", "qt", "dens")}
        hydro = [[fld() for _ in range(n)] for n in nhydro_records]
        scal = [fld() for _ in range(nscal)]
        buoy = ksgs = None
        if ivers > 0:
            if ivers <= 2:
                buoy = fld()
            if with_dif:
                ksgs = fld()
    return Restart(header, profiles, fields, scal, hydro, buoy, ksgs, vers)
