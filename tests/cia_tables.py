"""Synthetic HITRAN CIA tables for the tests (the HITRAN tables are not redistributable).

Written in the .cia layout the reader expects: a header line per block
("pair  nu_min  nu_max  N  T  sigma_max ...") followed by "nu sigma" lines."""
import numpy as np


def blocks_n2():
    """N2-N2: one band, 3 temperatures; the 250 K block stored in descending nu with a
    negative value (clamped to 0 when read)."""
    out = []
    for T, scale in ((200.0, 1.3), (250.0, 1.1), (300.0, 0.9)):
        nu = np.linspace(695.0, 712.0, 35)
        sg = scale * 2.0e-45 * np.exp(-((nu - 703.0) / 4.0) ** 2)
        out.append((T, nu, sg))
    return out


def blocks_o2(n=20):
    """O2-O2: n blocks at n temperatures over the same range (more than the 16 the device
    caches per grid point)."""
    return [(180.0 + 7.0 * k, np.linspace(690.0, 715.0, 26), (1.0 + 0.03 * k) * 8.0e-46 * np.ones(26))
            for k in range(n)]


def blocks_co2():
    """CO2-CO2: two disjoint bands at two temperatures each (nu outside both -> 0)."""
    out = []
    for lo, hi in ((696.0, 700.0), (705.0, 709.5)):
        for T in (220.0, 290.0):
            nu = np.linspace(lo, hi, 17)
            out.append((T, nu, (T / 250.0) * 3.0e-43 * (1.0 + 0.1 * np.sin(nu))))
    return out


def write_cia(path, pair, blocks, descending=(), negative=()):
    lines = []
    for k, (T, nu, sg) in enumerate(blocks):
        nu, sg = np.asarray(nu), np.array(sg)
        if k in negative:
            sg[len(sg) // 2] = -1.0e-48
        if k in descending:
            nu, sg = nu[::-1], sg[::-1]
        lines.append(f"{pair:>20}{nu.min():10.3f}{nu.max():10.3f}{len(nu):7d}{T:7.1f}{sg.max():10.3E}"
                     f"{0.0:6.3f}{'synthetic':>27}")
        lines += [f"{a:10.4f} {b:10.3E}" for a, b in zip(nu, sg)]
    path.write_text("\n".join(lines) + "\n")


def loaded(blocks, negative=()):
    """What the reader returns for `blocks` (values as written with 4 significant digits)."""
    out = []
    for k, (T, nu, sg) in enumerate(blocks):
        nu = np.array([float(f"{a:10.4f}") for a in nu])
        sg = np.array([float(f"{b:10.3E}") for b in sg])
        if k in negative:
            sg[len(sg) // 2] = 0.0
        out.append((T, nu, sg))
    return out
