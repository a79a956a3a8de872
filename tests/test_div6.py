"""The pressure stencils divide by six with a reciprocal and one fused remainder correction (Brisebarre, Muller
and Raina, 2004) where x is a normal float of at least 2^-120, and by IEEE division elsewhere. The method is a
property of IEEE single-precision arithmetic, so it is checked here on the host CPU with the same float
operations (fmaf is the fused multiply-add the device uses): every significand at eight exponents of both signs,
the floats around the guard, subnormals, zeros, infinities and NaN must give IEEE x / 6 bit for bit. The device
kernels are held to the same floats by the solver's parity tests."""

import shutil
import subprocess
from pathlib import Path

import pytest

SOURCE = Path(__file__).resolve().parent / "native" / "div6_check.c"


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_division_by_six_is_ieee_division(tmp_path):
    exe = tmp_path / "div6_check"
    # -ffp-contract=off: only the written fmaf calls fuse; -mfma: fmaf is one hardware instruction
    flags = ["-O2", "-ffp-contract=off", "-fno-fast-math"]
    build = subprocess.run(["gcc", *flags, "-mfma", "-o", str(exe), str(SOURCE), "-lm"], capture_output=True, text=True)
    if build.returncode != 0:  # a host without FMA instructions still has a correctly rounded libm fmaf
        build = subprocess.run(["gcc", *flags, "-o", str(exe), str(SOURCE), "-lm"], capture_output=True, text=True)
    assert build.returncode == 0, build.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    bad, checked = int(out[0]), int(out[1])
    assert checked > 150_000_000
    assert bad == 0, f"{bad} of {checked} quotients differ from IEEE division"
