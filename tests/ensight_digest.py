"""Digest of an Ensight ASCII file with round-off noise removed.

The reference's non-regression check is a byte comparison of its Ensight
files (6 significant digits).  Values at the level of round-off differ
between any two summation orders, so the digest is taken of a canonical
text: values below a floor (relative to the file's largest magnitude)
become zero, and the time in ensight.case keeps 12 significant digits.
Fields made mostly of cancellations -- the node velocity of a shock tube,
whose transverse components and precursor are round-off, and the
pseudo-viscosity -- are compared to 3 significant digits above 1e-6 of
their largest value; every other field byte for byte above 1e-10.  The
header and connectivity text always match byte for byte.
"""
import hashlib
import os

COARSE = ("Velocity", "PseudoViscosity")


def _is_value(s: str) -> bool:
    return "e" in s and s.replace("e", "").replace(".", "").replace("-", "").replace("+", "").isdigit()


def canonical(text: str, coarse: bool = False) -> str:
    lines = text.split("\n")
    vals = [abs(float(ln)) for ln in lines if _is_value(ln.strip())]
    floor = (1e-6 if coarse else 1e-10) * max(vals) if vals else 0.
    out = []
    after_time = False
    for ln in lines:
        s = ln.strip()
        if after_time and s:
            out.append(f"{float(s):.12g}")
            after_time = False
            continue
        if s == "time values:":
            after_time = True
        if _is_value(s):
            v = float(s)
            if abs(v) <= floor:
                v = 0.
            ln = f"{v:12.2e}" if coarse else (ln if v != 0. else f"{0.0:12.5e}")
        out.append(ln)
    return "\n".join(out)


def digest(path: str) -> str:
    coarse = os.path.basename(os.path.dirname(path)) in COARSE
    return hashlib.sha256(canonical(open(path).read(), coarse).encode()).hexdigest()
