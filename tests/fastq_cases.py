"""Seeded FASTQ chunk buffers for the parse tests: well-formed chunks and
every way the reference's reader (src/read.c:11-63) stops early -- a missing
'@' or '+', an empty sequence, a quality of another length, a chunk without
its last newline, blank lines after it, CR line ends, a NUL inside, and two
files of different read counts."""
from __future__ import annotations

import numpy as np

BASES = np.frombuffer(b"ACGTNacgt", np.uint8)


def _record(rng, i: int, mate: int, seq_len: int, opts: dict) -> bytes:
    name = opts.get("name", f"r{i}/{mate}".encode())
    s = BASES[rng.integers(0, 9 if opts.get("mixed") else 4, seq_len)].tobytes()
    qlen = seq_len + opts.get("qual_delta", 0)
    q = (np.full(max(qlen, 0), 33, np.uint8) + rng.integers(0, 41, max(qlen, 0)).astype(np.uint8)).tobytes()
    plus = opts.get("plus", b"+")
    eol = b"\r\n" if opts.get("cr") else b"\n"
    if opts.get("cr"):
        # a CR is part of the line for the reference: keep lengths equal
        q = q[:-1] if q else q
    return b"@" + name + eol + s + eol + plus + eol + q + b"\n"


def chunk(rng, n: int, mate: int = 1, bad: str = "", at: int = -1, lens=(1, 320),
          cr: bool = False, mixed: bool = False) -> bytes:
    """n records; `bad` spoils record `at` (or the chunk's end)."""
    out = []
    for i in range(n):
        L = int(rng.integers(lens[0], lens[1] + 1))
        opts = {"cr": cr, "mixed": mixed}
        if rng.random() < 0.2:
            opts["plus"] = b"+" + f"r{i}/{mate}".encode()
        if rng.random() < 0.05:
            opts["name"] = b""
        if i == at:
            if bad == "no_at":
                out.append(b"X" + _record(rng, i, mate, L, opts)[1:])
                continue
            if bad == "no_plus":
                opts["plus"] = b"-"
            elif bad == "empty_seq":
                L = 0
            elif bad == "qual_long":
                opts["qual_delta"] = 1
            elif bad == "qual_short":
                opts["qual_delta"] = -1
        out.append(_record(rng, i, mate, L, opts))
    b = b"".join(out)
    if bad == "no_last_newline" and b:
        b = b[:-1]
    elif bad == "blank_tail":
        b = b + b"\n" * int(rng.integers(1, 3))
    elif bad == "nul_inside" and b:
        k = int(rng.integers(0, len(b)))
        b = b[:k] + b"\0" + b[k + 1:]
    elif bad == "truncated" and b:
        b = b[:int(rng.integers(1, len(b)))]
    elif bad == "garbage_tail":
        b = b + b"junk"
    return b


BAD = ["", "", "", "no_at", "no_plus", "empty_seq", "qual_long", "qual_short", "no_last_newline",
       "blank_tail", "nul_inside", "truncated", "garbage_tail"]


def pair_cases(seed: int, count: int, max_n: int = 40, max_len: int = 320):
    """(left, right) buffers of assorted shapes."""
    rng = np.random.default_rng(seed)
    cases = [(b"", b""), (b"", b"@a\nA\n+\nI\n"), (b"@a\nA\n+\nI\n", b""), (b"@a\nA\n+\nI", b"@a\nA\n+\nI\n")]
    for _ in range(count):
        nl = int(rng.integers(1, max_n))
        nr = nl if rng.random() < 0.6 else int(rng.integers(1, max_n))
        bl = "" if rng.random() < 0.6 else BAD[int(rng.integers(0, len(BAD)))]
        br = "" if rng.random() < 0.6 else BAD[int(rng.integers(0, len(BAD)))]
        cr = rng.random() < 0.1
        mixed = rng.random() < 0.3
        lens = (1, max_len) if rng.random() < 0.5 else (min(50, max_len), min(150, max_len))
        left = chunk(rng, nl, 1, bl, int(rng.integers(0, nl)), lens, cr, mixed)
        right = chunk(rng, nr, 2, br, int(rng.integers(0, nr)), lens, cr, mixed)
        cases.append((left, right))
    return cases


def single_cases(seed: int, count: int, max_n: int = 40, max_len: int = 320):
    rng = np.random.default_rng(seed)
    cases = [b"", b"@a\nA\n+\nI", b"@\nAC\n+\nII\n\n"]
    for _ in range(count):
        n = int(rng.integers(1, max_n))
        cases.append(chunk(rng, n, 1, BAD[int(rng.integers(0, len(BAD)))], int(rng.integers(0, n)),
                           (1, max_len), rng.random() < 0.1, rng.random() < 0.3))
    return cases
