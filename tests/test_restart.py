"""The reference's restart file format (src/IO/restarting.f90 savedata :778-1068): CPU
checks of fdd3260_b200.restart against a record-by-record construction of the bytes
savedata's WRITE statements produce (4-byte length markers around each record, items
packed, real(8), integer(4))."""
import struct

import numpy as np
import pytest

from fdd3260_b200 import restart


def _rec(b):
    return struct.pack("<i", len(b)) + b + struct.pack("<i", len(b))


def _tiny(nscal=2, ksgs=True):
    nx, ny, nz = 6, 7, 5
    rng = np.random.default_rng(1)
    sh = (nz, ny, nx)
    hdr = {"time": 123.5, "ntime": 42, "dt": 0.75, "ntau": 1, "nx": nx, "ny": ny, "nz": nz, "dx": 25.0, "dy": 30.0,
           "dz": 10.0, "nscal": nscal, "nparc": 0, "xn_ccn0": 1e8, "xn_in0": 0.0}
    prof = {k: rng.normal(size=nz) for k in restart.PROFILES}
    prof["scal0"] = rng.normal(size=(nscal, nz))
    flds = {k: rng.normal(size=sh) for k in ("u", "v", "w", "p", "es", "qt", "dens")}
    scal = [rng.normal(size=sh) for _ in range(nscal)]
    return restart.Restart(hdr, prof, flds, scal, ksgs=rng.normal(size=sh) if ksgs else None)


def test_bytes_match_savedata_records(tmp_path):
    r = _tiny()
    path = tmp_path / "restart.dat"
    restart.write(str(path), r)
    h = r.header
    want = _rec(b"V04")
    want += _rec(struct.pack("<didiiiidddiidd", h["time"], h["ntime"], h["dt"], h["ntau"], h["nx"], h["ny"], h["nz"],
                             h["dx"], h["dy"], h["dz"], h["nscal"], h["nparc"], h["xn_ccn0"], h["xn_in0"]))
    # u00 ... k0, then scal0(1:nz, 1:nscal) column-major
    want += _rec(b"".join(r.profiles[k].astype("<f8").tobytes() for k in restart.PROFILES) +
                 np.asfortranarray(r.profiles["scal0"].T).tobytes(order="F"))
    for k in ("u", "v", "w", "p", "es", "qt", "dens"):
        # x(1:nx,1:ny,1:nz) column-major == the (nz, ny, nx) C-ordered array
        want += _rec(np.asfortranarray(np.transpose(r.fields[k], (2, 1, 0))).tobytes(order="F"))
    for a in r.scal:
        want += _rec(a.tobytes())
    want += _rec(r.ksgs.tobytes())
    assert path.read_bytes() == want
    assert len(want[8:8 + 3]) == 3 and struct.unpack("<i", want[11:15])[0] == 84   # header record: 84 bytes


def test_round_trip(tmp_path):
    r = _tiny(nscal=3)
    path = str(tmp_path / "r.dat")
    restart.write(path, r)
    q = restart.read(path, with_dif=True)
    assert q.header == r.header and q.vers == b"V04"
    for k in restart.PROFILES + ["scal0"]:
        assert np.array_equal(q.profiles[k], r.profiles[k])
    for k in r.fields:
        assert np.array_equal(q.fields[k], r.fields[k])
    assert all(np.array_equal(a, b) for a, b in zip(q.scal, r.scal))
    assert np.array_equal(q.ksgs, r.ksgs)


def test_old_versions_and_framing_errors(tmp_path):
    r = _tiny(nscal=1, ksgs=False)
    r.vers = b"V02"
    r.buoy = np.ones((5, 7, 6))
    path = str(tmp_path / "v2.dat")
    restart.write(path, r)
    q = restart.read(path, with_dif=False)
    assert np.array_equal(q.buoy, r.buoy) and q.ksgs is None
    # a truncated file fails loudly
    data = open(path, "rb").read()
    open(path, "wb").write(data[:-5])
    with pytest.raises((ValueError, EOFError, struct.error)):
        restart.read(path)


def test_oversize_record_rejected(tmp_path, monkeypatch):
    monkeypatch.setattr(restart, "MAX_RECORD", 100)
    with pytest.raises(ValueError):
        restart.write(str(tmp_path / "x.dat"), _tiny())
