"""Write a `Scene` as a SolTrace .stinput system file.

The format is the one the SolTrace CLI reads (coretrace/strace/main.cpp:78-397) and
`st_b200_load_stinput` reads: a version line, the sun (point source flag, shape, sigma or
half-width, position, user sunshape table), the optical property pairs (one tab-separated
line per face with an optional reflectivity / transmissivity table after it), then the
stages and their elements (29 tab-separated fields per element).  Numbers are written with
Python's shortest round-trip repr, so the file reads back to the same doubles.
"""
from __future__ import annotations

from .scenes import OpticFace, Scene


def _n(x) -> str:
    return repr(float(x))


def _face(f: OpticFace) -> list:
    rt, tt = f.refl_table, f.trans_table
    line = "\t".join(["OPTICAL", f.dist[:1], "0", "1", "0", _n(f.refl), _n(f.trans), _n(f.slope), _n(f.spec),
                      _n(f.n_real), _n(f.n_imag), "0", "0", "0", "0",
                      "1" if rt else "0", str(len(rt[0]) if rt else 0),
                      "1" if tt else "0", str(len(tt[0]) if tt else 0)])
    out = [line]
    for tab in (rt, tt):
        if tab:
            out += [f"{_n(a)} {_n(v)}" for a, v in zip(tab[0], tab[1])]
    return out


def _pad8(v) -> list:
    v = list(v)[:8]
    return [_n(x) for x in v + [0.0] * (8 - len(v))]


def stinput_text(sc: Scene, version: str = "3.1.0") -> str:
    s = sc.sun
    lines = [f"# SOLTRACE VERSION {version} INPUT FILE",
             "\t".join(["SUN", "PTSRC", "1" if s.point_source else "0", "SHAPE", s.shape[:1],
                        "SIGMA", _n(s.sigma), "HALFWIDTH", _n(s.sigma)]),
             "\t".join(["XYZ", *map(_n, s.xyz), "USELDH", "0", "LDH", "0", "0", "0"])]
    table = s.table
    lines.append(f"USER SHAPE DATA\t{len(table[0]) if table else 0}")
    if table:
        lines += [f"{_n(a)}\t{_n(i)}" for a, i in zip(table[0], table[1])]
    lines.append(f"OPTICS LIST COUNT\t{len(sc.optics)}")
    for o in sc.optics:
        lines.append(f"OPTICAL PAIR\t{o.name}")
        lines += _face(o.front) + _face(o.back)
    lines.append(f"STAGE LIST COUNT\t{len(sc.stages)}")
    for k, st in enumerate(sc.stages):
        lines.append("\t".join(["STAGE", "XYZ", *map(_n, st.origin), "AIM", *map(_n, st.aim), "ZROT", _n(st.zrot),
                                "VIRTUAL", str(int(st.virtual)), "MULTIHIT", str(int(st.multihit)),
                                "ELEMENTS", str(len(st.elements)), "TRACETHROUGH", str(int(st.tracethrough))]))
        lines.append(f"Stage {k + 1}")
        for e in st.elements:
            lines.append("\t".join([str(int(e.enabled)), *map(_n, e.origin), *map(_n, e.aim), _n(e.zrot),
                                    e.aperture[:1], *_pad8(e.aperture_params), e.surface[:1],
                                    *_pad8(e.surface_params), e.surface_file or "", e.optic, str(int(e.interaction))]))
    return "\n".join(lines) + "\n"


def write_stinput(sc: Scene, path: str) -> str:
    with open(path, "w") as f:
        f.write(stinput_text(sc))
    return path
