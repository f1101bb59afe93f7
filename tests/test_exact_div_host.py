"""The certified division of csrc/exact_div.cuh, built for the host
(tests/exact_div_host.cpp) and checked against IEEE division bit for bit.

The device path refines the hardware reciprocal estimate, then accepts a
quotient only when an exact residual shows it is RN(a/b); everything else goes
to the IEEE operator.  Here the estimate is replaced by 1/b with a relative
error up to 0.2, so the certification itself is what keeps the results exact:
no mismatch is allowed for any estimate, and the counts show that the fast
path takes nearly every in-range quotient once the estimate is as good as the
hardware's (about 2^-23) and almost none when it is useless.  The GPU's own
estimate is covered by a3g_selftest_div on the device.
"""
import pathlib
import shutil
import subprocess

import pytest

HERE = pathlib.Path(__file__).resolve().parent


@pytest.fixture(scope="module")
def results(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ is not available")
    exe = tmp_path_factory.mktemp("exact_div") / "exact_div_host"
    subprocess.check_call([gxx, "-O2", "-std=c++17", "-ffp-contract=off", "-o", str(exe),
                           str(HERE / "exact_div_host.cpp")])
    out = subprocess.run([str(exe), "200000", "3"], capture_output=True, text=True, timeout=300)
    rows = {}
    for line in out.stdout.splitlines():
        f = line.split()
        if len(f) == 9 and f[3] == "pairs":
            rows[(f[0], f[1], float(f[2]))] = dict(n=int(f[4]), bad=int(f[6]), fallbacks=int(f[8]))
    assert out.returncode == 0, out.stdout[-2000:]
    assert len(rows) == 50
    return rows


def test_every_quotient_is_ieee(results):
    bad = {k: v["bad"] for k, v in results.items() if v["bad"]}
    assert not bad


def test_fast_path_takes_in_range_quotients(results):
    # limiter-like ratios: only power-of-two quotients fall back (a zero dividend is a*b)
    for rel in (0.0, 1.2e-7, 6.0e-5):
        r = results[("div_rn", "limiter", rel)]
        assert r["fallbacks"] < 0.002 * r["n"], (rel, r)


def test_poor_estimates_fall_back(results):
    # a 20 % estimate defeats the iteration: the IEEE operator answers, still exactly
    for fam in ("wide", "near_exact", "limiter", "tails", "special"):
        r = results[("div_rn", fam, 0.2)]
        assert r["fallbacks"] > 0.9 * r["n"], (fam, r)
    # out-of-range operands always take the IEEE operator
    assert results[("div_rn", "wide", 0.0)]["fallbacks"] > 0.1 * 200000


def test_tails_take_the_fast_path(results):
    # dividends down a diffused cloud's tail over pivots in [1, 4): the back
    # substitution's fast path certifies every dividend of 2^-900 and above
    # (81 % of the family's exponents, -1080 .. -150); the rest, down to the
    # subnormals, goes to the IEEE operator
    r = results[("div_rn_rcp", "tails", 0.0)]
    assert r["bad"] == 0
    assert 0.15 * r["n"] < r["fallbacks"] < 0.23 * r["n"], r
