"""The command line fastfib [n] [--print] against the reference's
tests/cli.ps1:9-32 cases: argument order, --print and --help, n read from
stdin, the 64-bit edge (F(93) is the last Fibonacci number below 2^64), and
status 1 with a message for bad input.  Bad input is rejected before the GPU
is touched, so those cases run on the CPU; the cases that compute run on the
GPU, plus the digits of F(10^6) against the reference-generated hash."""
import hashlib
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "fastfib_b200", "fastfib")

# (arguments, stdin or None, exit status, text the output must contain, text it must not)
COMPUTE = [
    ("10 --print", None, 0, "fibonacci(10) = 55", None),
    ("--print 10", None, 0, "fibonacci(10) = 55", None),
    ("0 --print", None, 0, "fibonacci(0) = 0", None),
    ("1 --print", None, 0, "fibonacci(1) = 1", None),
    ("2 --print", None, 0, "fibonacci(2) = 1", None),
    ("93 --print", None, 0, "fibonacci(93) = 12200160415121876738", None),
    ("94 --print", None, 0, "fibonacci(94) = 19740274219868223167", None),
    ("007 --print", None, 0, "fibonacci(7) = 13", None),
    ("1000", None, 0, "Time:", "fibonacci("),
    ("--print", "12", 0, "fibonacci(12) = 144", None),
    ("--print", "  12  ", 0, "fibonacci(12) = 144", None),
]
REJECT = [
    ("--help", None, 0, "usage: fastfib", None),
    ("-h", None, 0, "usage: fastfib", None),
    ("--print", "abc", 1, "invalid n: abc", None),
    ("--print", "", 1, "invalid n", None),
    ("-5", None, 1, "invalid argument: -5", None),
    ("+5", None, 1, "invalid argument: +5", None),
    ("1e9", None, 1, "invalid argument: 1e9", None),
    ("0x10", None, 1, "invalid argument: 0x10", None),
    ("18446744073709551616", None, 1, "invalid argument", None),
    ("10 20", None, 1, "invalid argument: 20", None),
    ("--bogus", None, 1, "usage: fastfib", None),
]


@pytest.fixture(scope="module")
def cli():
    from fastfib_b200.build import build
    build()
    assert os.path.exists(CLI)
    return CLI


def run(cli, args, stdin):
    r = subprocess.run([cli, *args.split()], input=(stdin + "\n") if stdin is not None else None,
                       capture_output=True, text=True, timeout=300)
    return r.returncode, r.stdout + r.stderr


@pytest.mark.parametrize("args,stdin,code,expect,reject", REJECT)
def test_rejects_and_help(cli, args, stdin, code, expect, reject):
    rc, text = run(cli, args, stdin)
    assert rc == code and expect in text, (rc, text)


def test_cases_cover_the_reference_list():
    assert len(COMPUTE) + len(REJECT) == 22


@pytest.mark.gpu
@pytest.mark.parametrize("args,stdin,code,expect,reject", COMPUTE)
def test_compute(cli, args, stdin, code, expect, reject):
    rc, text = run(cli, args, stdin)
    assert rc == code and expect in text, (rc, text)
    assert reject is None or reject not in text


@pytest.mark.gpu
def test_digits_f1e6(cli):
    rc, text = run(cli, "1000000 --print", None)
    assert rc == 0
    line = next(l for l in text.splitlines() if l.startswith("fibonacci(1000000) = "))
    digits = line.split(" = ", 1)[1]
    with open(os.path.join(ROOT, "tests", "golden", "decimal_sha256.json")) as f:
        gold = json.load(f)
    assert hashlib.sha256(digits.encode()).hexdigest() == gold["1000000"]
    assert "Decimal conversion:" in text
