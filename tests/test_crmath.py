"""The correctly rounded exp and x^(1/4) of vhlle_b200/csrc/vh_crmath.cuh,
compiled for the host from the same header (IEEE operations and explicit
fma only, no contraction, so the host build gives the device's bits):
every result equals the exact value rounded to nearest (60-digit decimal
arithmetic), over random arguments and the edges (subnormal results,
overflow, tiny arguments)."""
import decimal
import math
import os
import subprocess
from fractions import Fraction

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "vhlle_b200", "csrc", "vh_crmath.cuh")

PROGRAM = r"""
#include <cstdio>
#include <cstdlib>
#include "vh_crmath.cuh"
int main() {
  char f[8];
  double x;
  while (std::scanf("%1s %la", f, &x) == 2) {
    const double y = f[0] == 'e' ? vh::crm::exp_cr(x) : vh::crm::root4_cr(x);
    std::printf("%a\n", y);
  }
  return 0;
}
"""


@pytest.fixture(scope="module")
def crm(tmp_path_factory):
    d = tmp_path_factory.mktemp("crm")
    src = d / "crm.cpp"
    src.write_text(PROGRAM)
    exe = d / "crm"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I",
                    os.path.dirname(HEADER), str(src), "-o", str(exe)], check=True)

    def run(kind, xs):
        inp = "".join("%s %s\n" % (kind, float(x).hex()) for x in xs)
        out = subprocess.run([str(exe)], input=inp, capture_output=True, text=True, check=True)
        return [float.fromhex(t) for t in out.stdout.split()]
    return run


decimal.getcontext().prec = 60


def correctly_rounded(y, exact):
    """y is the double nearest to the exact value (Decimal; inf allowed)."""
    if math.isinf(y):
        return exact > Fraction(2) ** 1024 - Fraction(2) ** 970
    ex = Fraction(exact)
    u = Fraction(math.ulp(y))
    d = abs(ex - Fraction(y))
    if y == 0.0:
        return ex <= Fraction(2) ** -1075
    # also allow y = the double just below a power of two boundary from above
    return d <= u / 2 or (d <= Fraction(math.ulp(math.nextafter(y, 0))) / 2)


def test_exp_is_correctly_rounded(crm):
    rng = np.random.default_rng(3)
    xs = list(rng.uniform(-1, 1, 1500)) + list(rng.uniform(-50, 50, 1500)) + \
        list(rng.uniform(-745.2, -700, 400)) + list(rng.uniform(700, 709.78, 200)) + \
        list(rng.uniform(-1e-6, 1e-6, 200)) + \
        [0.0, -0.0, 1.0, -1.0, 709.782712893384, 709.79, -745.13321910194, -745.1332191019412,
         -745.14, -708.3964185322641, -708.4, 1e-300, -1e-300, 5e-324]
    ys = crm("e", xs)
    bad = [(x, y) for x, y in zip(xs, ys) if not correctly_rounded(y, decimal.Decimal(x).exp())]
    assert not bad, bad[:5]
    assert crm("e", [float("nan")])[0] != crm("e", [float("nan")])[0]  # NaN
    assert crm("e", [800.0, -800.0]) == [float("inf"), 0.0]


def test_fourth_root_is_correctly_rounded(crm):
    rng = np.random.default_rng(4)
    xs = list(10 ** rng.uniform(-300, 300, 1000)) + list(10 ** rng.uniform(-3, 4, 2000)) + \
        [1.0, 16.0, 0.0625, 2.0, 5e-324, 1.7976931348623157e308]
    ys = crm("r", xs)
    bad = [(x, y) for x, y in zip(xs, ys)
           if not correctly_rounded(y, decimal.Decimal(x).sqrt().sqrt())]
    assert not bad, bad[:5]
    assert crm("r", [0.0, float("inf")]) == [0.0, float("inf")]
