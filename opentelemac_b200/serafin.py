"""SERAFIN / SELAFIN mesh and result files (TELEMAC's .slf format).

A SERAFIN file is a Fortran sequential unformatted file: every record is
framed by its byte length as a 4-byte integer before and after.  Records,
in order (sources/utils/hermes/utils_serafin.F; the reference's Python
reader scripts/python27/parsers/parserSELAFIN.py:502-600):

    TITLE             80 characters (the last 8 name the format: 'SERAFIN ' /
                      'SERAFIND' for double precision)
    NBV1, NBV2        numbers of variables and of "clandestine" variables
    NBV1+NBV2 names   32 characters each: 16 of name, 16 of unit
    IPARAM(10)        IPARAM(7) > 1: number of planes (3D); IPARAM(10) = 1:
                      a date record follows
    [DATE(6)]         year, month, day, hour, minute, second
    NELEM, NPOIN, NDP, 1
    IKLE              NELEM*NDP integers, element by element, 1-based
    IPOBO             NPOIN integers (boundary numbering, 0 inside)
    X, Y              NPOIN reals each
    per time step     TIME (one real), then one record of NPOIN reals per
                      variable

Reals are binary32 in SERAFIN and binary64 in SERAFIND files; files are
big-endian as TELEMAC writes them, and the reader also accepts
little-endian ones (detected from the title record's length, as the
reference reader does).  The float width is detected from the length of
the X record.
"""
import numpy as np


class Serafin:
    """Contents of a SERAFIN file.  ikle is 0-based, shape (nelem, ndp)."""

    def __init__(self, title="", var_names=(), var_units=(), iparam=None, date=None,
                 ikle=None, ipobo=None, x=None, y=None, times=(), values=(), double=False,
                 endian=">", nbv2=0):
        self.title = title
        self.var_names = list(var_names)
        self.var_units = list(var_units)
        self.nbv2 = nbv2
        self.iparam = np.zeros(10, dtype=np.int64) if iparam is None else np.asarray(iparam)
        self.date = None if date is None else np.asarray(date)
        self.ikle = None if ikle is None else np.asarray(ikle)
        self.ipobo = ipobo
        self.x = x
        self.y = y
        self.times = list(times)
        self.values = list(values)       # per time step: (nvar, npoin) array
        self.double = double
        self.endian = endian

    @property
    def npoin(self):
        return int(self.x.size)

    @property
    def nelem(self):
        return int(self.ikle.shape[0])

    @property
    def ndp(self):
        return int(self.ikle.shape[1])

    def ikle_fortran(self):
        """IKLE(NELEM, NDP) column-major, 1-based: BIEF_MESH's layout."""
        return np.ascontiguousarray((self.ikle.T + 1).astype(np.int32)).ravel()


class _Reader:
    def __init__(self, buf):
        self.buf = buf
        self.pos = 0
        self.endian = ">"

    def record(self):
        if self.pos + 4 > len(self.buf):
            raise EOFError
        n = int(np.frombuffer(self.buf, dtype=self.endian + "i4", count=1, offset=self.pos)[0])
        start = self.pos + 4
        end = start + n
        if n < 0 or end + 4 > len(self.buf):
            raise ValueError("truncated SERAFIN record")
        tail = int(np.frombuffer(self.buf, dtype=self.endian + "i4", count=1, offset=end)[0])
        if tail != n:
            raise ValueError("corrupt SERAFIN record markers")
        self.pos = end + 4
        return start, n

    def ints(self):
        start, n = self.record()
        return np.frombuffer(self.buf, dtype=self.endian + "i4", count=n // 4, offset=start)

    def chars(self):
        start, n = self.record()
        return bytes(self.buf[start:start + n])


def read(path, values=True):
    """Read a SERAFIN file.  values=False stops after the mesh (geometry
    files have no time steps anyway)."""
    with open(path, "rb") as fh:
        buf = fh.read()
    r = _Reader(buf)
    head = int(np.frombuffer(buf, dtype=">i4", count=1)[0]) if len(buf) >= 4 else 0
    r.endian = ">" if head == 80 else "<"
    title = r.chars().decode("latin-1")
    nbv = r.ints()
    nbv1, nbv2 = int(nbv[0]), int(nbv[1])
    names, units = [], []
    for _ in range(nbv1 + nbv2):
        c = r.chars().decode("latin-1")
        names.append(c[:16].rstrip())
        units.append(c[16:32].rstrip())
    iparam = np.array(r.ints(), dtype=np.int64)
    date = np.array(r.ints(), dtype=np.int64) if iparam[9] == 1 else None
    dims = r.ints()
    nelem, npoin, ndp = int(dims[0]), int(dims[1]), int(dims[2])
    ikle = np.array(r.ints(), dtype=np.int64).reshape(nelem, ndp) - 1
    ipobo = np.array(r.ints(), dtype=np.int64)
    start, n = r.record()
    width = n // npoin
    if width not in (4, 8) or width * npoin != n:
        raise ValueError("cannot tell the float width of the X record")
    ftype = np.dtype(r.endian + ("f8" if width == 8 else "f4"))
    x = np.frombuffer(buf, dtype=ftype, count=npoin, offset=start).astype(np.float64)
    start, _ = r.record()
    y = np.frombuffer(buf, dtype=ftype, count=npoin, offset=start).astype(np.float64)
    out = Serafin(title=title, var_names=names[:nbv1], var_units=units[:nbv1], iparam=iparam,
                  date=date, ikle=ikle, ipobo=ipobo, x=x, y=y, double=(width == 8),
                  endian=r.endian, nbv2=nbv2)
    out.var_names_all = names
    out.var_units_all = units
    if not values:
        return out
    nvar = nbv1 + nbv2
    while r.pos < len(buf):
        try:
            start, _ = r.record()
        except EOFError:
            break
        t = float(np.frombuffer(buf, dtype=ftype, count=1, offset=start)[0])
        frame = np.empty((nvar, npoin))
        for v in range(nvar):
            start, _ = r.record()
            frame[v] = np.frombuffer(buf, dtype=ftype, count=npoin, offset=start)
        out.times.append(t)
        out.values.append(frame)
    return out


def _rec(parts, payload, endian):
    n = np.array([len(payload)], dtype=endian + "i4").tobytes()
    parts.extend([n, payload, n])


def write(path, s):
    """Write a Serafin object (big-endian unless s.endian is '<';
    SERAFIND when s.double)."""
    e = s.endian
    ftype = np.dtype(e + ("f8" if s.double else "f4"))
    parts = []
    title = s.title.encode("latin-1")
    if len(title) != 80:     # a new title: 72 characters and the format tag
        title = title[:72].ljust(72) + (b"SERAFIND" if s.double else b"SERAFIN ")
    _rec(parts, title, e)
    names = list(s.var_names) + list(getattr(s, "var_names_all", s.var_names)[len(s.var_names):])
    units = list(s.var_units) + list(getattr(s, "var_units_all", s.var_units)[len(s.var_units):])
    _rec(parts, np.array([len(s.var_names), s.nbv2], dtype=e + "i4").tobytes(), e)
    for nm, un in zip(names, units):
        _rec(parts, nm.encode("latin-1")[:16].ljust(16) + un.encode("latin-1")[:16].ljust(16), e)
    iparam = np.array(s.iparam, dtype=e + "i4").copy()
    iparam[9] = 1 if s.date is not None else 0
    _rec(parts, iparam.tobytes(), e)
    if s.date is not None:
        _rec(parts, np.array(s.date, dtype=e + "i4").tobytes(), e)
    _rec(parts, np.array([s.nelem, s.npoin, s.ndp, 1], dtype=e + "i4").tobytes(), e)
    _rec(parts, (np.asarray(s.ikle) + 1).astype(e + "i4").tobytes(), e)
    ipobo = np.zeros(s.npoin, dtype=np.int64) if s.ipobo is None else np.asarray(s.ipobo)
    _rec(parts, ipobo.astype(e + "i4").tobytes(), e)
    _rec(parts, np.asarray(s.x).astype(ftype).tobytes(), e)
    _rec(parts, np.asarray(s.y).astype(ftype).tobytes(), e)
    for t, frame in zip(s.times, s.values):
        _rec(parts, np.array([t]).astype(ftype).tobytes(), e)
        for row in np.asarray(frame):
            _rec(parts, np.asarray(row).astype(ftype).tobytes(), e)
    with open(path, "wb") as fh:
        fh.write(b"".join(parts))


def mesh_file(path, x, y, ikle0, title="B200 BIEF mesh", double=True):
    """Write a geometry-only SERAFIN file for a P1 mesh."""
    write(path, Serafin(title=title, ikle=np.asarray(ikle0), x=np.asarray(x),
                        y=np.asarray(y), double=double))
