"""Synthetic IASI L1C EPS-native granules for the tests: the record framing and field
offsets of the format (as runtests.jl:528-566 of IRSounderLBL.jl writes them)."""
import numpy as np

MDR_SIZE = 2728908


def _grh(cls, sub, size):
    g = np.zeros(20, np.uint8)
    g[0] = g[1] = cls
    g[2] = sub
    g[3:7] = np.frombuffer(np.array([size], ">u4").tobytes(), np.uint8)
    return g


def _put(buf, off, arr, dt):
    b = np.ascontiguousarray(np.asarray(arr), dtype=dt).tobytes()
    buf[off:off + len(b)] = np.frombuffer(b, np.uint8)


def write_nat(path, l1c, n_mdr=1, raw=None, geo=None, exponent=7):
    """raw: int16 [n_mdr, 120, 8700] spectra (default 7000 everywhere, i.e. 70 mW radiance at
    exponent 7); geo(q, s, p, line) -> (lon, lat, zen, azi, sza, saa, cld, lnd)."""
    mphr_p = np.frombuffer(b"INSTRUMENT_ID = IASI\nSPACECRAFT_ID = M02\n", np.uint8)
    parts = [np.concatenate([_grh(1, 0, 20 + len(mphr_p)), mphr_p])]
    giadr = np.concatenate([_grh(5, 1, 84), np.zeros(64, np.uint8)])
    _put(giadr, 20, [1], ">i2")
    _put(giadr, 22, [1], ">i2")
    _put(giadr, 42, [8700], ">i2")
    _put(giadr, 62, [exponent], ">i2")
    parts.append(giadr)
    for m in range(n_mdr):
        mdr = np.zeros(MDR_SIZE, np.uint8)
        mdr[:20] = _grh(8, 2, MDR_SIZE)
        _put(mdr, l1c.OFF_NSFIRST, [1], ">i4")
        _put(mdr, l1c.OFF_NSLAST, [8461], ">i4")
        g = np.zeros((120, 8))
        for s in range(30):
            for p in range(4):
                q = 4 * s + p
                g[q] = geo(q, s, p, m) if geo else (-120.0 - q * 0.001, 30.0 + q * 0.002, 5.0 + p,
                                                      100.0 + q * 0.05, 40.0 + s * 0.1, 160.0 - q * 0.1, q % 101, 50)
        _put(mdr, l1c.OFF_GEOLOC, np.round(g[:, [0, 1]] / 1e-6).astype(np.int64).ravel(), ">i4")
        _put(mdr, l1c.OFF_ANG_SAT, np.round(g[:, [2, 3]] / 1e-6).astype(np.int64).ravel(), ">i4")
        _put(mdr, l1c.OFF_ANG_SUN, np.round(g[:, [4, 5]] / 1e-6).astype(np.int64).ravel(), ">i4")
        mdr[l1c.OFF_CLDFRAC:l1c.OFF_CLDFRAC + 120] = g[:, 6].astype(np.uint8)
        mdr[l1c.OFF_LNDFRAC:l1c.OFF_LNDFRAC + 120] = g[:, 7].astype(np.uint8)
        spec = np.full((120, 8700), 7000, np.int16) if raw is None else raw[m]
        _put(mdr, l1c.OFF_SPEC, spec.ravel(), ">i2")
        parts.append(mdr)
    with open(path, "wb") as f:
        for p in parts:
            f.write(p.tobytes())
