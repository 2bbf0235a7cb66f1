"""Seeded random parameter files in the three driver formats, and runs of the
reference's own parsers on them (oracle/_ref/params_ref_<format>, built by
oracle/Makefile from TESTS/sequential/io.cpp, TESTS/parallel/io_par.cpp and
TESTS/hypre/pargemslr_hypre_interface.cpp).

Each format is a list of line kinds, read off those parsers: a keyword line
takes one word from a fixed list; an "N<k>" line takes up to k numbers.  The
files vary what the parsers are sensitive to: keyword case, unknown keywords,
fewer or more numbers than a line takes (a trailing comment that starts with
a number is then read as one), exponent markers without digits, truncated
files, extra lines and lines longer than the 1023-byte read buffer.  Keyword
lines always end with a space and a comment and hold no tabs: the reference
reads a keyword up to a space only, and past the end of a line that has none.
"""
from __future__ import annotations

import os
import random
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")

B = ["ILUT", "ILUK", "GEMSLR"]
C4 = ["ILUT", "ILUK", "BJILUT", "BJILUK"]
C6 = C4 + ["BJILUT2", "BJILUK2"]
GP = ["BJ", "ESCHUR", "GEMSLR", "PSLR"]
PART = ["ND", "RKWAY"]
REORD = ["NO", "RCM", "AMD", "ND"]
LR = ["STD", "TR", "SUB"]
SOLVE3 = ["LU", "U", "MUL"]
SOLVE2 = ["LU", "U"]
SMOOTH = ["MILU", "ILU"]

FORMATS = {
    "sequential": [B, "N1", B] + ["N1"] * 8 + [PART, PART] + ["N1"] * 6 + [REORD, LR, LR] + ["N1"] * 14
                  + [SOLVE3, "N1"],
    "parallel": [GP, "N1", B, "N1", B, C6] + ["N1"] * 5 + ["N2", "N2", PART, PART, "N4", "N3", "N3", REORD,
                                                          LR, LR, LR] + ["N3"] * 5 + ["N1"] * 4
                + [SOLVE3, "N3", "N3", "N1"],
    "hypre": [GP, "N1", B, "N1", B, C4, "N1", "N2", "N2", PART, PART, "N4", "N3", "N3", REORD, LR, LR]
             + ["N2"] * 5 + ["N1"] * 4 + [SOLVE2, "N1", "N1", SMOOTH, "N1"],
}
assert [len(v) for v in FORMATS.values()] == [38, 35, 31]

ALL_WORDS = sorted({w for v in FORMATS.values() for k in v if isinstance(k, list) for w in k})
PLAIN_NUMBERS = ["5", "-3", "0", "200", "1.5", ".25", "2.", "-0.0", "1e-03", "2.5E+2", "1e8", "-7.125e-1",
                 "3.0", "0.001", "12345678"]
ODD_NUMBERS = ["1e", "3E+", "7e-", "4ergs", "1-2", "1..2", "-", "+", "abc", "5e5e"]


def _case(rng: random.Random, w: str) -> str:
    r = rng.random()
    return w if r < 0.6 else (w.lower() if r < 0.8 else "".join(c.lower() if rng.random() < 0.5 else c for c in w))


def _comment(rng: random.Random, k: int) -> str:
    return rng.choice([f"{k}. name = text", "name = text", f"{k + 3} words after", "(x, y)"])


def _line(rng: random.Random, kind, k: int) -> str:
    lead = " " * rng.randint(0, 3)
    if isinstance(kind, list):
        r = rng.random()
        if r < 0.975:
            w = _case(rng, rng.choice(kind))
        elif r < 0.9875:
            w = rng.choice(ALL_WORDS)
        else:
            w = rng.choice(["ILUX", "GEMSLRX", "LUU"])
        return f"{lead}{w}{' ' * rng.randint(1, 20)}{_comment(rng, k)}\n"
    want = int(kind[1:])
    r = rng.random()
    m = want if r < 0.7 else (rng.randint(0, want - 1) if r < 0.85 else want + rng.randint(1, 2))
    toks = [rng.choice(ODD_NUMBERS if rng.random() < 0.08 else PLAIN_NUMBERS) for _ in range(m)]
    sep = lambda: rng.choice([" ", "  ", "   ", "\t", " \t "])  # noqa: E731
    body = "".join(t + sep() for t in toks)
    if rng.random() < 0.05:
        body = "word " + body
    return f"{lead}{body}{' ' * rng.randint(1, 8)}{_comment(rng, k)}\n"


def random_file(fmt: str, seed: int) -> str:
    rng = random.Random(seed * 7919 + len(fmt))
    kinds = FORMATS[fmt]
    n = len(kinds)
    r = rng.random()
    if r < 0.15:
        n = rng.randint(0, len(kinds) - 1)
    lines = [_line(rng, kinds[i], i + 1) for i in range(n)]
    if r > 0.85:
        lines += [_line(rng, rng.choice(["N1", B]), n + j + 1) for j in range(rng.randint(1, 3))]
    if lines and rng.random() < 0.05:
        i = rng.randrange(len(lines))
        lines[i] = lines[i][:-1] + " " + " ".join("w" * rng.randint(1, 9) for _ in range(260)) + " x \n"
    return "".join(lines)


def reference_available(fmt: str) -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"params_ref_{fmt}"))


def run_reference(fmt: str, path: str, fill: float | None = None):
    """(status, 180 values) from the reference parser of `fmt` on the file."""
    cmd = [os.path.join(REF_DIR, f"params_ref_{fmt}"), path] + ([repr(float(fill))] if fill is not None else [])
    out = subprocess.run(cmd, capture_output=True, text=True, check=True).stdout.split("\n")
    k = max(i for i, line in enumerate(out) if line.startswith("rc "))  # after the parser's own messages
    rc = int(out[k].split()[1])
    vals = np.array([float.fromhex(line.split()[1]) for line in out[k + 1:k + 181]])
    return rc, vals


def run_reference_args(argv):
    """(status, 180 values) from the sequential driver's read_inputs on argv, over the defaults."""
    cmd = [os.path.join(REF_DIR, "params_ref_sequential"), "--args", *argv]
    out = subprocess.run(cmd, capture_output=True, text=True, check=True).stdout.split("\n")
    k = max(i for i, line in enumerate(out) if line.startswith("rc "))
    return int(out[k].split()[1]), np.array([float.fromhex(line.split()[1]) for line in out[k + 1:k + 181]])
