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


def test_shared_reciprocal_division_in_the_normal_range(tmp_path):
    """A division by a shared reciprocal, RN32(RN64(x * r)) with r within one f64
    ulp of 1/y, equals the IEEE quotient wherever |x / y| >= 2^-126; below that an
    exact quotient can be a midpoint of the subnormal grid (the check finds such
    pairs), so a kernel using it must keep the IEEE division there
    (tests/native/recip_division_check.c)."""
    exe = str(tmp_path / "recip_division_check")
    subprocess.run(["gcc", "-O2", "-fopenmp", "-ffp-contract=off", os.path.join(ROOT, "tests", "native", "recip_division_check.c"),
                    "-o", exe, "-lm"], check=True)
    out = subprocess.run([exe, str(1 << 24)], capture_output=True, text=True, check=True).stdout.split()
    checked, bad, bad_normal = int(out[0]), int(out[1]), int(out[2])
    assert checked > (1 << 24)
    assert bad_normal == 0, out
    assert bad > 0  # the subnormal-grid ties exist, which is why the range limit is needed
