"""The CUDA smoothstep divides by the difference of its two literal edges with a
Markstein-corrected reciprocal product instead of the IEEE division; this proves
the two equal for every divisor the kernels use, over the whole range the
kernels route through the short sequence (2^-100 <= |x| <= 2^100), by checking
every float in it (tests/native/divconst_check.c)."""
import glob
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "fenix_b200", "csrc")
CALL = re.compile(r"smoothstepv\(([^,]*),([^,]*),")
LITERAL = re.compile(r"^\s*(-?[0-9]+\.?[0-9]*)f\s*$")


def call_sites():
    out = []
    for path in sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cuh"))):
        for n, line in enumerate(open(path), 1):
            if "FX_DEV" in line and "smoothstepv(" in line:
                continue  # a definition
            for m in CALL.finditer(line):
                out.append((os.path.basename(path), n, m.group(1), m.group(2)))
    return out


def test_every_smoothstep_call_has_literal_edges():
    bad = [s for s in call_sites() if not (LITERAL.match(s[2]) and LITERAL.match(s[3]))]
    assert not bad, f"smoothstepv with edges that are not f32 literals (use smoothstep_dyn): {bad}"


def test_constant_divisions_equal_ieee_division(tmp_path):
    exe = str(tmp_path / "divconst_check")
    subprocess.run(["gcc", "-O2", "-mfma", "-fopenmp", "-ffp-contract=off", os.path.join(ROOT, "tests", "native", "divconst_check.c"),
                    "-o", exe, "-lm"], check=True)
    divisors = sorted({float(np.float32(float(LITERAL.match(e1).group(1))) - np.float32(float(LITERAL.match(e0).group(1))))
                       for _, _, e0, e1 in call_sites()})
    assert len(divisors) >= 20
    out = subprocess.run([exe] + [d.hex() for d in divisors], capture_output=True, text=True, check=True).stdout.split("\n")
    rows = [r.split() for r in out if r.strip()]
    assert len(rows) == len(divisors)
    failures = [r for r in rows if int(r[1]) != 0]
    assert not failures, f"divisors whose short sequence differs from IEEE division: {failures}"
