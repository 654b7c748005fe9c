"""Tiny FITS reader/writer for the tests (primary + IMAGE HDUs only)."""
from __future__ import annotations

import numpy as np

_DT = {8: ">u1", 16: ">i2", 32: ">i4", 64: ">i8", -32: ">f4", -64: ">f8"}


def read_fits(path: str):
    """List of (header dict, flat float64 data) per HDU."""
    b = open(path, "rb").read()
    off = 0
    hdus = []
    while off + 2880 <= len(b):
        cards = []
        while True:
            blk = b[off:off + 2880]
            off += 2880
            cs = [blk[i * 80:(i + 1) * 80].decode("ascii") for i in range(36)]
            cards += cs
            if any(c.startswith("END ") for c in cs):
                break
        kv = {}
        for c in cards:
            if c[8:10] == "= ":
                v = c[10:].split("/")[0].strip()
                kv[c[:8].strip()] = v.strip("'").strip() if v.startswith("'") else v
        bp = int(kv["BITPIX"])
        na = int(kv["NAXIS"])
        shape = [int(kv["NAXIS%d" % i]) for i in range(1, na + 1)]
        n = int(np.prod(shape)) if na else 0
        nb = n * abs(bp) // 8
        d = np.frombuffer(b[off:off + nb], dtype=_DT[bp]).astype(np.float64)
        bscale = float(kv.get("BSCALE", 1.0))
        bzero = float(kv.get("BZERO", 0.0))
        if bscale != 1.0 or bzero != 0.0:
            d = d * bscale + bzero
        off += (nb + 2879) // 2880 * 2880
        kv["_cards"] = cards
        hdus.append((kv, d))
    return hdus


def write_header_only(path: str, header: str) -> None:
    """Header cards (80-char, with END) followed by a zero data unit."""
    assert len(header) % 80 == 0
    cards = [header[i:i + 80] for i in range(0, len(header), 80)]
    kv = {c[:8].strip(): c[10:].split("/")[0].strip() for c in cards if c[8:10] == "= "}
    bp = int(kv["BITPIX"])
    n = 1
    for i in range(1, int(kv["NAXIS"]) + 1):
        n *= int(kv["NAXIS%d" % i])
    h = header.encode("ascii")
    h += b" " * ((-len(h)) % 2880)
    nb = n * abs(bp) // 8
    with open(path, "wb") as f:
        f.write(h)
        f.write(b"\0" * (nb + (-nb) % 2880))


def write_input_map(path: str, values: np.ndarray, lon: np.ndarray, lat: np.ndarray) -> None:
    """Input map in the reference's layout (HCGrid/gmap.cpp:102-148):
    primary image NAXIS1=1, NAXIS2=N[, NAXIS3=C] of float32 values, then an
    IMAGE extension NAXIS1=N, NAXIS2=2 holding lon then lat (float64)."""
    values = np.asarray(values, np.float32).reshape(-1, len(lon))
    nchan, n = values.shape

    def card(k, v):
        return ("%-8s= %20s" % (k, v)).ljust(80)

    h = [card("SIMPLE", "T"), card("BITPIX", -32), card("NAXIS", 3 if nchan > 1 else 2), card("NAXIS1", 1),
         card("NAXIS2", n)] + ([card("NAXIS3", nchan)] if nchan > 1 else []) + [card("EXTEND", "T"), "END".ljust(80)]
    e = [("%-8s= %-20s" % ("XTENSION", "'IMAGE   '")).ljust(80), card("BITPIX", -64), card("NAXIS", 2),
         card("NAXIS1", n), card("NAXIS2", 2), card("PCOUNT", 0), card("GCOUNT", 1), "END".ljust(80)]

    def block(b):
        return b + b"\0" * ((-len(b)) % 2880)

    def hblock(cards):
        s = "".join(cards).encode("ascii")
        return s + b" " * ((-len(s)) % 2880)

    with open(path, "wb") as f:
        f.write(hblock(h))
        f.write(block(values.astype(">f4").tobytes()))
        f.write(hblock(e))
        f.write(block(np.concatenate([lon, lat]).astype(">f8").tobytes()))
